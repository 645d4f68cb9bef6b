"""Shared builders for the parity tests."""
import numpy as np


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    d = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (d if d > 0 else 1.0)


def mixed_geometry(nx, ny, nz, seed=5, walls=True, solid_block=True, biofilm=True):
    """A small map with every material class: pore 2, wall 1, solid 0 (NoDynamics on the flow
    lattice), two biofilm codes 3 and 4; ghost planes duplicate their neighbours."""
    rng = np.random.default_rng(seed)
    m = np.full((nx, ny, nz), 2, np.int8)
    inner = m[1:-1]
    for _ in range(4):
        c = rng.integers([0, 0, 0], [nx - 2, ny, nz])
        r = rng.uniform(1.5, 2.8)
        X, Y, Z = np.ogrid[:nx - 2, :ny, :nz]
        inner[(X - c[0]) ** 2 + (Y - c[1]) ** 2 + (Z - c[2]) ** 2 <= r * r] = 1
    if solid_block:
        inner[nx // 3:nx // 3 + 2, ny // 2 - 1:ny // 2 + 1, 1:3] = 0
    if biofilm:
        inner[(rng.random(inner.shape) < 0.05) & (inner == 2)] = 3
        inner[(rng.random(inner.shape) < 0.03) & (inner == 2)] = 4
    if walls:
        m[:, 0, :] = m[:, -1, :] = 1
        m[:, :, 0] = m[:, :, -1] = 1
    m[0] = m[1]
    m[-1] = m[-2]
    return m.ravel()
