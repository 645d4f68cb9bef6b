"""Writes tests/golden/diagnostics.json: seeded diagnostic rows run through the reference's own
complab_diag::Diagnostics (complab3d_diagnostics.hh, compiled into oracle/_ref/libref_diag.so by
`make -C oracle ref`), with the CSV it wrote and its messages and final report.

Run from the repository root in a checkout that has the reference sources:
    make -C oracle ref && python tests/golden/make_golden_diag.py
"""
import ctypes as C
import json
import os
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))


def case(L, rng, tol, exprs, names, n_rows, drift, negative):
    nf = len(names)
    iters = np.arange(n_rows, dtype=np.int64) * 500
    por = rng.uniform(0.3, 0.5, n_rows)
    opened = rng.integers(1000, 5000, n_rows).astype(np.int64)
    base = rng.uniform(0.1, 10.0, (1, nf, 5))
    stats = np.repeat(base, n_rows, axis=0)
    stats[:, :, 2] = np.abs(stats[:, :, 2])
    for r in range(1, n_rows):
        stats[r, :, 0] *= 1.0 + drift * r * rng.uniform(-1, 1, nf)
    if negative:
        stats[n_rows // 2, 0, 2] = -3e-9
    stats = np.ascontiguousarray(stats)
    csv = os.path.join(tempfile.mkdtemp(), "summary.csv")
    ce = (C.c_char_p * max(1, len(exprs)))(*[e.encode() for e in exprs])
    cn = (C.c_char_p * nf)(*[n.encode() for n in names])
    msgs, rep = C.create_string_buffer(1 << 16), C.create_string_buffer(1 << 14)
    P = lambda a: a.ctypes.data_as(C.c_void_p)
    L.ref_diag_run(csv.encode(), C.c_double(tol), len(exprs), ce, n_rows, nf, cn, P(iters), P(por), P(opened),
                   P(stats), msgs, len(msgs), rep, len(rep))
    return dict(tol=tol, exprs=exprs, names=names, iterations=iters.tolist(), porosity=por.tolist(),
                open_voxels=opened.tolist(), stats=stats.tolist(), csv=open(csv).read(),
                messages=msgs.value.decode(), report=rep.value.decode().replace(csv, "<csv>"))


def main():
    L = C.CDLL(os.path.join(ROOT, "oracle", "_ref", "libref_diag.so"))
    rng = np.random.default_rng(11)
    cases = [case(L, rng, 1e-6, ["Fe2+FeS", "HS+FeS"], ["Fe2", "HS", "FeS"], 6, 0.0, False),
             case(L, rng, 1e-6, ["Fe2+FeS", "Ca"], ["Fe2", "HS", "FeS"], 5, 1e-4, True),
             case(L, rng, 1e-3, ["A+B", "B"], ["A", "B", "mic"], 7, 1e-5, False),
             case(L, rng, 1e-6, ["A"], ["A", "B"], 1, 0.0, False),
             case(L, rng, 1e-6, [], ["A"], 3, 0.0, True)]
    with open(os.path.join(ROOT, "tests", "golden", "diagnostics.json"), "w") as f:
        json.dump(cases, f)
    print(f"wrote {len(cases)} diagnostics cases")


if __name__ == "__main__":
    main()
