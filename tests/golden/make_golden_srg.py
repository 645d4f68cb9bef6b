"""Writes the seeded surrogate networks of tests/golden/srg (.srg files in the reference's format,
complab3d_surrogate.hh) and tests/golden/srg.json: the reference's own evaluation of each (load()
and Network::evalAll() after evalBound's clamp to the training box), compiled into
oracle/_ref/libref_srg.so by `make -C oracle ref REFSRC=<CompLaB3D-GEMS checkout>`. Every network
is evaluated on seeded input rows, some outside its training box.

    python tests/golden/make_golden_srg.py
"""
import ctypes as C
import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
SRG = os.path.join(HERE, "srg")

# name, input names (None: positional), layer sizes, logoutput, output scale, training box
NETWORKS = [
    ("uptake_growth.srg", ["A", "B"], [2, 10, 10, 3], 0, 0.2, (0.0, 50.0)),
    ("log_growth.srg", ["B", "C", "A"], [3, 8, 1], 1, 1.0, (0.0, 20.0)),
    ("positional.srg", None, [2, 6, 6, 1], 0, 0.1, (0.0, 30.0)),
    ("largest.srg", ["A", "B", "C", "D", "E", "F", "G", "H"], [8, 32, 32, 32, 4], 0, 0.5, (0.0, 10.0)),
]


def fmt(v):
    return " ".join(repr(float(x)) for x in np.ravel(v))


def write_network(path, names, sizes, logout, scale, box, seed):
    rng = np.random.default_rng(seed)
    n_in, n_out = sizes[0], sizes[-1]
    lo = np.full(n_in, box[0])
    hi = np.full(n_in, box[1]) * rng.uniform(0.6, 1.0, n_in)
    lines = ["# seeded surrogate network for the tests (not trained)", "version 1", f"inputs {n_in}",
             "layers " + " ".join(str(s) for s in sizes), f"logoutput {logout}"]
    if names:
        lines.append("inputnames " + " ".join(names))
    lines += ["xoffset " + fmt(lo), "xgain " + fmt(2.0 / (hi - lo)), "xymin -1", f"outputs {n_out}",
              "outputnames growth" + "".join(f" r_{k}" for k in range(1, n_out)),
              "yoffset " + fmt(np.r_[(-1.0 if logout else 0.0), -scale * rng.uniform(0, 1, n_out - 1)]),
              "ygain " + fmt(2.0 / (scale * rng.uniform(1.0, 2.0, n_out))), "yymin -1",
              "trainmin " + fmt(lo), "trainmax " + fmt(hi),
              "outrange" + "".join(f" 0 {scale}" for _ in range(n_out))]
    for l in range(len(sizes) - 1):
        rows, cols = sizes[l + 1], sizes[l]
        W = rng.normal(0.0, 1.2 / np.sqrt(cols), size=(rows, cols))
        lines.append(f"W {l}")
        lines += [fmt(W[r]) for r in range(rows)]
        lines.append(f"B {l}")
        lines.append(fmt(rng.normal(0.0, 0.4, rows)))
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")
    return lo, hi


def main():
    L = C.CDLL(os.path.join(ROOT, "oracle", "_ref", "libref_srg.so"))
    L.ref_srg_info.argtypes = [C.c_char_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.c_char_p, C.c_int]
    L.ref_srg_eval.argtypes = [C.c_char_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.POINTER(C.c_long)]
    os.makedirs(SRG, exist_ok=True)
    out = []
    for k, (name, names, sizes, logout, scale, box) in enumerate(NETWORKS):
        path = os.path.join(SRG, name)
        lo, hi = write_network(path, names, sizes, logout, scale, box, 600 + k)
        ni, no = C.c_int(), C.c_int()
        msg = C.create_string_buffer(1024)
        if L.ref_srg_info(path.encode(), C.byref(ni), C.byref(no), msg, 1024) != 0:
            raise SystemExit(f"{path}: {msg.value.decode()}")
        rng = np.random.default_rng(700 + k)
        n = 64
        X = rng.uniform(lo, hi, size=(n, ni.value))
        X[::8] = lo - 0.2 * (hi - lo)
        X[3::8] = hi * 1.5
        X = np.ascontiguousarray(X)
        Y = np.zeros((n, no.value))
        clamped = C.c_long()
        if L.ref_srg_eval(path.encode(), n, X.ctypes.data, 1, Y.ctypes.data, C.byref(clamped)) != 0:
            raise SystemExit(f"{path}: evaluation failed")
        out.append({"file": name, "inputs": names, "x": X.tolist(), "out": Y.tolist(), "clamped_rows": clamped.value})
        print(name, "inputs", ni.value, "outputs", no.value, "clamped rows", clamped.value)
    with open(os.path.join(HERE, "srg.json"), "w") as f:
        json.dump(out, f)


if __name__ == "__main__":
    main()
