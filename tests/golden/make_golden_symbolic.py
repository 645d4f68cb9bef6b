"""Writes tests/golden/symbolic.json: the reference's own evaluation of the rate-law files in
tests/golden/sym (complab3d_symbolic.hh: load() with its derived reaction lines, evaluate() with the
range clamp and the unit scale), compiled into oracle/_ref/libref_symbolic.so by
`make -C oracle ref REFSRC=<CompLaB3D-GEMS checkout>`. Each file is evaluated on seeded variable
rows, some of them outside the file's ranges and some at zero or negative values, so the guards
(division by zero, logarithms and roots of non-positive numbers) are exercised.

    python tests/golden/make_golden_symbolic.py
"""
import ctypes as C
import glob
import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))


def main():
    L = C.CDLL(os.path.join(ROOT, "oracle", "_ref", "libref_symbolic.so"))
    L.ref_sym_info.argtypes = [C.c_char_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.c_char_p, C.c_int]
    L.ref_sym_eval.argtypes = [C.c_char_p, C.c_int, C.c_void_p, C.c_void_p, C.POINTER(C.c_long)]
    out = []
    for k, path in enumerate(sorted(glob.glob(os.path.join(HERE, "sym", "*.sym")))):
        nv, nr = C.c_int(), C.c_int()
        names = C.create_string_buffer(4096)
        if L.ref_sym_info(path.encode(), C.byref(nv), C.byref(nr), names, 4096) != 0:
            raise SystemExit(f"{path}: {names.value.decode()}")
        rng = np.random.default_rng(100 + k)
        n = 64
        X = 10.0 ** rng.uniform(-4, 0.7, size=(n, nv.value))
        X[::7] *= -1.0                      # negative values (below a range, or guarded functions)
        X[3::9] = 0.0                       # exact zeros
        X[5::11] *= 40.0                    # far above a range
        X = np.ascontiguousarray(X)
        Y = np.zeros((n, nr.value))
        clamped = C.c_long()
        if L.ref_sym_eval(path.encode(), n, X.ctypes.data, Y.ctypes.data, C.byref(clamped)) != 0:
            raise SystemExit(f"{path}: evaluation failed")
        out.append({"file": os.path.basename(path), "n_vars": nv.value, "rates": names.value.decode().split(),
                    "vars": X.tolist(), "rates_out": Y.tolist(), "clamped_rows": clamped.value})
        print(os.path.basename(path), nv.value, names.value.decode(), "clamped rows", clamped.value)
    with open(os.path.join(HERE, "symbolic.json"), "w") as f:
        json.dump(out, f)


if __name__ == "__main__":
    main()
