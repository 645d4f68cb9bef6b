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


def test_truncated_file_leaves_the_handle_unchanged(clb, tmp_path):
    """A load that fails part-way (the file ends early) changes nothing: the step counters, the
    populations and the concentrations are those the handle had before the call."""
    shape = (14, 8, 7)
    mat = mixed_geometry(*shape, seed=3)
    bio = np.zeros((2, mat.size))
    A = setup(clb, mat, shape, clb.F64, bio)
    A.flow_step(11)
    A.couple_velocity()
    A.ade_step(9)
    path = os.path.join(tmp_path, "full.chk")
    A.checkpoint_save(path)
    assert not os.path.exists(path + ".tmp")
    raw = open(path, "rb").read()
    B = setup(clb, mat, shape, clb.F64, bio)
    B.flow_step(4)
    B.couple_velocity()
    B.ade_step(5)
    before = state(B)
    for cut in (len(raw) - 8, len(raw) // 2, 200):
        short = os.path.join(tmp_path, f"cut{cut}.chk")
        open(short, "wb").write(raw[:cut])
        with pytest.raises(clb.ClbError, match="truncated|not a checkpoint"):
            B.checkpoint_load(short)
        for a, b in zip(before, state(B)):
            np.testing.assert_array_equal(a, b)
    # one more step runs from the unchanged state at the unchanged parity
    C = setup(clb, mat, shape, clb.F64, bio)
    C.flow_step(4)
    C.couple_velocity()
    C.ade_step(5)
    B.ade_step(3)
    C.ade_step(3)
    np.testing.assert_array_equal(B.concentration(0), C.concentration(0))


def test_load_refuses_a_different_mobile_set(clb, tmp_path):
    """Two handles with the same species and microbe counts but mobile and immobile species
    swapped: the blocks would have different sizes, so the load is refused."""
    shape = (12, 8, 7)
    mat = mixed_geometry(*shape, seed=5)
    sp_a = [dict(omega_pore=1.0, left_type=1, right_type=1, c0=0.1),
            dict(omega_pore=1.0, mobile=0, left_type=1, right_type=1, c0=0.2)]
    sp_b = [dict(omega_pore=1.0, mobile=0, left_type=1, right_type=1, c0=0.1),
            dict(omega_pore=1.0, left_type=1, right_type=1, c0=0.2)]
    A = clb.Domain(mat, *shape, 0.8, flow_precision=clb.F64, ade_precision=clb.F64)
    A.flow_init(3e-4)
    A.ade_init(sp_a)
    path = os.path.join(tmp_path, "m.chk")
    A.checkpoint_save(path)
    B = clb.Domain(mat, *shape, 0.8, flow_precision=clb.F64, ade_precision=clb.F64)
    B.flow_init(3e-4)
    B.ade_init(sp_b)
    with pytest.raises(clb.ClbError, match="mobile species differ"):
        B.checkpoint_load(path)


def test_save_replaces_the_file_whole(clb, tmp_path):
    """Saving over an existing restart file goes through a temporary file and a rename: the old
    file stays readable until the new one is complete, and no temporary file is left behind."""
    shape = (12, 8, 7)
    mat = mixed_geometry(*shape, seed=6)
    D = clb.Domain(mat, *shape, 0.8, flow_precision=clb.F64)
    D.flow_init(3e-4)
    path = os.path.join(tmp_path, "r.chk")
    D.checkpoint_save(path, transport=False)
    D.flow_step(3)
    D.checkpoint_save(path, transport=False)
    assert sorted(os.listdir(tmp_path)) == ["r.chk"]
    E = clb.Domain(mat, *shape, 0.8, flow_precision=clb.F64)
    E.flow_init(3e-4)
    E.checkpoint_load(path)
    np.testing.assert_array_equal(E.flow_populations(), D.flow_populations())
