"""The straight-duct A + B -> C case of the reference's analytic check
(ABC_sweep_package/tools/analytic_channel.py), shared by the GPU test and the oracle's CPU test.

A duct of 34 x-planes with walls on the four side faces, three species A, B, C of one diffusivity
with every x face held (Dirichlet A = 1, B = 0, C = 0 at x = 0 and A = 0, B = 1, C = 0 at
x = nx - 1), the reaction A + B -> C at rate k A B (the library's CLB_LAW_PRECIP law with a mobile
product), and three unreacting tracer species fed with the boundary values of A - B, A + C and
B + C. A uniform velocity U along x sets Pe = U (nx - 1) / D."""
import json
import os

import numpy as np

NX, NY, NZ = 34, 8, 8
TAU = 1.5                 # D = (tau - 1/2) / 4 = 0.25
D = 0.25 * (TAU - 0.5)
K_REACT = 0.01            # k L^2 / D = 44: the reaction front is sharp, the clamp never binds
GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "channel.json")))


def material():
    m = np.full((NX, NY, NZ), 2, np.int8)
    m[:, 0, :] = m[:, -1, :] = 1
    m[:, :, 0] = m[:, :, -1] = 1
    return m.ravel()


def species():
    def sp(left, right):
        return dict(omega_pore=1.0 / TAU, omega_biofilm=1.0 / TAU, left_type=0, right_type=0,
                    left_bc=left, right_bc=right, c0=0.0)
    A0, B0 = GOLD["A0"], GOLD["B0"]
    return [sp(A0, 0.0), sp(0.0, B0), sp(0.0, 0.0),          # A, B, C
            sp(A0, -B0), sp(A0, 0.0), sp(0.0, B0)]           # tracers of A - B, A + C, B + C


def velocity(pe):
    u = np.zeros((3, NX * NY * NZ))
    u[0] = pe * D / (NX - 1)
    return u


ABIOTIC = [K_REACT, 0, 1, 2]   # rate k, reactants A (0) and B (1), product C (2)


def combinations(c):
    """The reaction-free combinations from the species fields c[s][N]."""
    A, B, C = c[0], c[1], c[2]
    return {"A - B": A - B, "A + C": A + C, "B + C": B + C}


def cross_section_mean(field):
    """One number per x-plane over the pore voxels of the plane (analytic_channel.cross_section_mean)."""
    pore = (material() == 2).reshape(NX, NY, NZ)
    f = np.asarray(field).reshape(NX, NY, NZ)
    return np.array([f[i][pore[i]].mean() for i in range(NX)])


def golden(pe, name):
    for c in GOLD["cases"]:
        if c["peclet"] == pe and c["combination"] == name:
            return np.array(c["profile"])
    raise KeyError((pe, name))
