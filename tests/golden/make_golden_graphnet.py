"""Writes the seeded graph networks of tests/golden/gnn (.gnn files in the reference's format,
complab3d_graphnet.hh) and tests/golden/graphnet.json: the reference's own evaluation of each
(load() and Network::eval() with the training-box clamp and the unit scale), compiled into
oracle/_ref/libref_graphnet.so by `make -C oracle ref REFSRC=<CompLaB3D-GEMS checkout>`. Every
network is evaluated on seeded concentration rows, some below or above its training box. Where the
checkout is named by CLB_REFERENCE_SRC, the reference's own example network
(examples/18_graph_network/input/aom.gnn) is evaluated too and recorded by its path in the checkout.

    CLB_REFERENCE_SRC=<checkout> python tests/golden/make_golden_graphnet.py
"""
import ctypes as C
import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
GNN = os.path.join(HERE, "gnn")

# name, species, reactions (stoichiometry rows = species), width, rounds, readout, growth, units,
# training box, output scale
NETWORKS = [
    ("extent_growth.gnn", ["A", "B", "C", "D"], [[-1, 0], [-1, -2], [1, 1], [0, 1]], 6, 2, "extent", 1, "per_hour",
     (0.0, 1.5), 2e-3),
    ("species_growth.gnn", ["A", "B", "C"], [[-1, 0.5], [0, -1], [2, 0]], 8, 3, "species", 1, "per_second",
     (0.0, 1.5), 1e-3),
    ("abiotic_extent.gnn", ["B", "C", "D"], [[-1], [1], [1]], 5, 1, "extent", 0, "per_second", (0.0, 1.5), 5e-4),
    ("largest_species.gnn", ["A", "B", "C", "D", "E"], [[-1, 0, 1], [1, -1, 0], [0, 1, -1], [2, 0, 0], [0, 0, 1]],
     16, 4, "species", 0, "per_second", (1e-5, 1e-2), 1e-6),
]


def fmt(v):
    return " ".join(repr(float(x)) for x in np.ravel(v))


def write_network(path, species, stoich, width, rounds, readout, growth, units, box, scale, seed):
    rng = np.random.default_rng(seed)
    S = np.asarray(stoich, dtype=float)
    nS, nR = S.shape
    W = width
    lo = np.full(nS, box[0]) + rng.uniform(0, 0.01 * (box[1] - box[0]), nS)
    hi = np.full(nS, box[1]) - rng.uniform(0, 0.01 * (box[1] - box[0]), nS)
    w = lambda *shape: rng.normal(0.0, 0.9 / np.sqrt(W), size=shape)  # noqa: E731
    lines = ["# seeded graph network for the tests (not trained)",
             f"provenance seed {seed}", "version 1", f"units {units}", "species " + " ".join(species),
             "reactions " + " ".join(f"R{r + 1}" for r in range(nR)), f"rounds {rounds}", f"width {W}",
             f"growth {growth}", f"readout {readout}", f"stoich {nS} {nR}"]
    lines += [fmt(S[i]) for i in range(nS)]
    lines.append("da " + fmt(rng.uniform(0.1, 2.0, nR)))
    lines.append("xoffset " + fmt(lo))
    lines.append("xgain " + fmt(2.0 / (hi - lo)))
    lines.append("xymin -1")
    n_y = (1 if growth else 0) if readout == "extent" else nS + (1 if growth else 0)
    if readout == "extent":
        lines.append("xiscale " + fmt(scale * rng.uniform(0.5, 1.5, nR)))
    if n_y:
        lines.append("yoffset " + fmt(-scale * rng.uniform(0.5, 1.5, n_y)))
        lines.append("ygain " + fmt(2.0 / (scale * rng.uniform(1.0, 3.0, n_y))))
    lines.append("yymin -1")
    lines.append("trainmin " + fmt(lo))
    lines.append("trainmax " + fmt(hi))
    lines.append("Wenc " + fmt(rng.normal(0.0, 1.0, W)))
    lines.append("benc " + fmt(rng.normal(0.0, 0.5, W)))
    for l in range(rounds):
        lines.append(f"layer {l}")
        lines.append("Wsr " + fmt(w(W, W)))
        lines.append("Wda " + fmt(rng.normal(0.0, 0.5, W)))
        lines.append("Wss " + fmt(w(W, W)))
        lines.append("Wrs " + fmt(w(W, W)))
        lines.append("bR " + fmt(rng.normal(0.0, 0.3, W)))
        lines.append("bS " + fmt(rng.normal(0.0, 0.3, W)))
    nh = 2 if growth else 1
    lines.append("Wout " + fmt(w(nh, W)))
    lines.append("bout " + fmt(rng.normal(0.0, 0.3, nh)))
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")
    return lo, hi


def evaluate(L, path, lo, hi, seed):
    ns, no = C.c_int(), C.c_int()
    msg = C.create_string_buffer(1024)
    if L.ref_gnn_info(path.encode(), C.byref(ns), C.byref(no), msg, 1024) != 0:
        raise SystemExit(f"{path}: {msg.value.decode()}")
    rng = np.random.default_rng(seed)
    n = 64
    X = rng.uniform(lo, hi, size=(n, ns.value))
    X[::9] = lo - 0.3 * (hi - lo)          # below the training box
    X[4::9] = hi + 0.7 * (hi - lo)         # above it
    X[7::13, 0] = 0.0
    X = np.ascontiguousarray(X)
    Y = np.zeros((n, no.value))
    clamped = C.c_long()
    if L.ref_gnn_eval(path.encode(), n, X.ctypes.data, Y.ctypes.data, C.byref(clamped)) != 0:
        raise SystemExit(f"{path}: evaluation failed")
    return X, Y, clamped.value


def main():
    L = C.CDLL(os.path.join(ROOT, "oracle", "_ref", "libref_graphnet.so"))
    L.ref_gnn_info.argtypes = [C.c_char_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.c_char_p, C.c_int]
    L.ref_gnn_eval.argtypes = [C.c_char_p, C.c_int, C.c_void_p, C.c_void_p, C.POINTER(C.c_long)]
    os.makedirs(GNN, exist_ok=True)
    out = []
    for k, (name, species, stoich, W, rounds, readout, growth, units, box, scale) in enumerate(NETWORKS):
        path = os.path.join(GNN, name)
        lo, hi = write_network(path, species, stoich, W, rounds, readout, growth, units, box, scale, 300 + k)
        X, Y, nc = evaluate(L, path, lo, hi, 400 + k)
        out.append({"file": name, "species": species, "growth": growth, "conc": X.tolist(), "out": Y.tolist(),
                    "clamped_rows": nc})
        print(name, "outputs", Y.shape[1], "clamped rows", nc)
    ref = os.environ.get("CLB_REFERENCE_SRC", "")
    example = os.path.join("examples", "18_graph_network", "input", "aom.gnn")
    if ref and os.path.isfile(os.path.join(ref, example)):
        # the example's own box, read from the file
        lo = hi = None
        for line in open(os.path.join(ref, example)):
            w = line.split()
            if w and w[0] == "trainmin":
                lo = np.array([float(v) for v in w[1:]])
            if w and w[0] == "trainmax":
                hi = np.array([float(v) for v in w[1:]])
        X, Y, nc = evaluate(L, os.path.join(ref, example), lo, hi, 500)
        out.append({"file": example, "in_reference_checkout": True, "conc": X.tolist(), "out": Y.tolist(),
                    "clamped_rows": nc})
        print(example, "outputs", Y.shape[1], "clamped rows", nc)
    with open(os.path.join(HERE, "graphnet.json"), "w") as f:
        json.dump(out, f)


if __name__ == "__main__":
    main()
