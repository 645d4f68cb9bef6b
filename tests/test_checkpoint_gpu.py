"""Restart files: a run saved mid-way (at an odd step count, so the AA parity is the odd one) and
loaded into a freshly set-up handle continues exactly as the uninterrupted run, bit for bit."""
import os

import numpy as np
import pytest

from helpers import mixed_geometry

pytestmark = pytest.mark.gpu

SPECIES = [
    dict(omega_pore=1 / 0.9, omega_biofilm=1 / 0.7, left_type=0, right_type=1, left_bc=1.0, c0=0.0),
    dict(omega_pore=1 / 0.62, omega_biofilm=1 / 0.56, left_type=1, right_type=0, right_bc=0.4, c0=0.2),
    dict(omega_pore=1.0, mobile=0, left_type=1, right_type=1, c0=0.3),
]


def setup(clb, mat, shape, prec, bio):
    D = clb.Domain(mat, *shape, 0.8, flow_precision=prec, ade_precision=prec, bio_codes=(3, 4), perm_ratio=(0.3, 0.3))
    D.flow_init(3e-4)
    D.ade_init(SPECIES)
    D.set_biomass(bio)
    D.set_kinetics(3, [1e-3, 0.1, 0.4, 1e-5], 1.0)
    return D


def state(D):
    out = [D.flow_populations()] + [D.concentration(s) for s in range(3)] + [D.biomass(m) for m in range(2)]
    return out


@pytest.mark.parametrize("prec", ["F64", "F32"])
def test_restart_continues_bit_for_bit(clb, tmp_path, prec):
    prec = getattr(clb, prec)
    shape = (16, 9, 8)
    mat = mixed_geometry(*shape, seed=4)
    rng = np.random.default_rng(2)
    bio = np.zeros((2, mat.size))
    bio[0, mat == 3] = rng.uniform(10, 60, size=(mat == 3).sum())
    bio[1, mat == 4] = rng.uniform(10, 60, size=(mat == 4).sum())
    A = setup(clb, mat, shape, prec, bio)
    A.flow_step(37)
    A.couple_velocity()
    A.ade_step(23)
    path = os.path.join(tmp_path, "run.chk")
    A.checkpoint_save(path)
    A.flow_step(19)
    A.ade_step(30)
    want = state(A)
    B = setup(clb, mat, shape, prec, np.zeros_like(bio))
    B.checkpoint_load(path)
    B.flow_step(19)
    B.ade_step(30)
    for a, b in zip(want, state(B)):
        np.testing.assert_array_equal(a, b)


def test_load_refuses_another_map(clb, tmp_path):
    shape = (12, 8, 7)
    mat = mixed_geometry(*shape, seed=1)
    D = clb.Domain(mat, *shape, 0.8)
    D.flow_init(3e-4)
    path = os.path.join(tmp_path, "f.chk")
    D.checkpoint_save(path, transport=False)
    other = mat.copy()
    other[np.flatnonzero(other == 2)[5]] = 0
    E = clb.Domain(other, *shape, 0.8)
    E.flow_init(3e-4)
    with pytest.raises(clb.ClbError):
        E.checkpoint_load(path)
    with pytest.raises(clb.ClbError):
        D.checkpoint_save(path, flow=False, transport=False)
