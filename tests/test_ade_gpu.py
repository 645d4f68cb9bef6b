"""Fused D3Q7 transport + kinetics on the GPU against the FP64 oracle."""
import numpy as np
import pytest

from helpers import mixed_geometry, rel_l2

pytestmark = pytest.mark.gpu

BIO = dict(bio_codes=(3, 4), perm_ratio=(0.3, 0.3))


def flow_field(oracle, mat, shape, steps=300):
    O = oracle.OracleFlow(mat, *shape, 0.8, 3e-4, bio_codes=(3, 4), perm_ratio=(0.3, 0.3))
    O.step(steps)
    return O.velocity()


def pair(clb, oracle, mat, shape, species, prec, u, law=0, params=(), dt=1.0, biomass=None):
    D = clb.Domain(mat, *shape, 0.8, ade_precision=prec, **BIO)
    D.ade_init(species)
    D.set_velocity(u)
    O = oracle.OracleAde(mat, *shape, species, u, bio_codes=(3, 4))
    if biomass is not None:
        D.set_biomass(biomass)
        O.set_biomass(biomass)
    if law:
        D.set_kinetics(law, params, dt)
        O.set_kinetics(law, params, dt)
    return D, O


SPECIES = [
    dict(omega_pore=1 / 0.9, omega_biofilm=1 / 0.7, left_type=0, right_type=1, left_bc=1.0, c0=0.0),
    dict(omega_pore=1 / 0.62, omega_biofilm=1 / 0.56, left_type=1, right_type=0, right_bc=0.4, c0=0.2),
    dict(omega_pore=1 / 1.3, omega_biofilm=1 / 0.9, left_type=2, right_type=2, c0=0.6),
]


@pytest.mark.parametrize("shape", [(20, 10, 9), (12, 8, 41)])
@pytest.mark.parametrize("steps", [1, 2, 25, 120])
def test_f64_multispecies_decay_matches_oracle(clb, oracle, shape, steps):
    mat = mixed_geometry(*shape)
    u = flow_field(oracle, mat, shape)
    D, O = pair(clb, oracle, mat, shape, SPECIES, clb.F64, u, law=1, params=[1e-3, 2e-2, 5e-3])
    D.ade_step(steps)
    O.step(steps)
    for s in range(3):
        pg, po = D.ade_populations(s), O.populations(s)
        assert np.max(np.abs(pg - po)) < 1e-12, s
        np.testing.assert_allclose(D.concentration(s), O.concentration(s), rtol=0, atol=1e-12)


def test_f64_monod_with_immobile_species(clb, oracle):
    shape = (16, 9, 8)
    mat = mixed_geometry(*shape, seed=3)
    u = flow_field(oracle, mat, shape)
    sp = SPECIES[:2] + [dict(omega_pore=1.0, mobile=0, left_type=1, right_type=1, c0=0.8)]
    D, O = pair(clb, oracle, mat, shape, sp, clb.F64, u, law=2, params=[1e-2, 3e-2, 1e-3, 0.1, 0.2, 0.5])
    D.ade_step(60)
    O.step(60)
    for s in range(3):
        np.testing.assert_allclose(D.concentration(s), O.concentration(s), rtol=0, atol=1e-12)


def test_f64_dual_monod_biomass(clb, oracle):
    shape = (16, 9, 8)
    mat = mixed_geometry(*shape, seed=4)
    u = flow_field(oracle, mat, shape)
    N = mat.size
    rng = np.random.default_rng(2)
    bio = np.zeros((2, N))
    bio[0, mat == 3] = rng.uniform(10, 60, size=(mat == 3).sum())
    bio[1, mat == 4] = rng.uniform(10, 60, size=(mat == 4).sum())
    D, O = pair(clb, oracle, mat, shape, SPECIES, clb.F64, u, law=3, params=[1e-3, 0.1, 0.4, 1e-5], biomass=bio)
    D.ade_step(80)
    O.step(80)
    for s in range(3):
        np.testing.assert_allclose(D.concentration(s), O.concentration(s), rtol=0, atol=1e-12)
    ob = O.biomass()
    for m in range(2):
        np.testing.assert_allclose(D.biomass(m), ob[m], rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("prec,tol", [("F32", 1e-5), ("F16S", 2e-2)])
def test_reduced_precision_concentration_error(clb, oracle, prec, tol):
    shape = (20, 10, 9)
    mat = mixed_geometry(*shape)
    u = flow_field(oracle, mat, shape)
    D, O = pair(clb, oracle, mat, shape, SPECIES, getattr(clb, prec), u, law=1, params=[1e-3, 2e-2, 5e-3])
    D.ade_step(200)
    O.step(200)
    for s in range(3):
        err = rel_l2(D.concentration(s), O.concentration(s))
        print(f"{prec} species {s} rel L2 {err:.3e}")
        assert err < tol


def test_closed_box_content_conserved_f64(clb, oracle):
    """A closed box with every reaction off: total + held (the reduction's content: every
    population of the lattice, walls included) is the conserved quantity, constant to 4e-13 relative
    as the reference states for it (README.md, summary CSV `_held`), over 1000 steps with flow. The
    reduction is a fixed-order FP64 tree, so asking twice gives the same bits."""
    shape = (18, 10, 9)
    mat = mixed_geometry(*shape)
    u = flow_field(oracle, mat, shape)
    sp = [dict(omega_pore=1 / 0.9, omega_biofilm=1 / 0.7, left_type=2, right_type=2, c0=0.3),
          dict(omega_pore=1 / 1.4, omega_biofilm=1 / 0.6, left_type=2, right_type=2, c0=1.7)]
    D, _ = pair(clb, oracle, mat, shape, sp, clb.F64, u)
    r0 = D.reduce()
    assert r0["content"].tobytes() == D.reduce()["content"].tobytes()
    D.ade_step(1000)
    r1 = D.reduce()
    r1b = D.reduce_noalloc()
    for key in ("total", "content", "min", "max"):
        assert r1[key].tobytes() == r1b[key].tobytes(), key
    drift = np.abs(r1["content"] - r0["content"]) / np.abs(r0["content"])
    assert np.all(drift <= 4e-13), drift
    # total alone is not conserved: mass resting in the walls moves in and out of it
    assert np.any(np.abs(r1["total"] - r0["total"]) > 1e-9 * np.abs(r0["total"]))


def test_coupled_velocity_equals_flow_velocity(clb):
    shape = (14, 8, 8)
    mat = mixed_geometry(*shape)
    D = clb.Domain(mat, *shape, 0.8, flow_precision=clb.F64, ade_precision=clb.F64, **BIO)
    D.flow_init(1e-4)
    D.flow_step(50)
    D.ade_init(SPECIES[:1])
    D.couple_velocity()
    u = np.empty(3 * D.N)
    lib = clb.lib()
    assert lib.clb_get_field(D.h, clb.FIELD_ADE_VELOCITY, 0, u.ctypes.data_as(clb.C.c_void_p), 0) == 0
    np.testing.assert_array_equal(u.reshape(3, -1), D.velocity())


@pytest.mark.parametrize("prec,n_species", [("F32", 6), ("F64", 3), ("F32", 2)])
def test_pipelined_step_matches_plain_bit_for_bit(clb, oracle, prec, n_species):
    """The pipelined transport step (next node's gathers in flight) does the same arithmetic as
    the plain one: identical populations and biomass after an odd number of steps."""
    shape = (22, 11, 10)
    mat = mixed_geometry(*shape, seed=6)
    u = flow_field(oracle, mat, shape)
    N = mat.size
    bio = np.zeros((2, N))
    bio[0, mat == 3] = 30.0
    bio[1, mat == 4] = 20.0
    species = [SPECIES[s % 3] for s in range(n_species)]
    out = []
    for pipe in (0, 1):
        D = clb.Domain(mat, *shape, 0.8, ade_precision=getattr(clb, prec), **BIO)
        D.tune("ade_pipe", pipe)
        D.ade_init(species)
        D.set_velocity(u)
        D.set_biomass(bio)
        D.set_kinetics(3, [1e-3, 0.1, 0.4, 1e-5], 1.0)
        D.ade_step(41)
        out.append([D.ade_populations(s) for s in range(n_species)] + [D.biomass(m) for m in range(2)])
    for a, b in zip(*out):
        np.testing.assert_array_equal(a, b)


def test_reductions_match_the_oracle_fields(clb, oracle):
    """clb_reduce over x = 1..nx-2 and the open (pore + biofilm) voxels (complab3d_processors_part3
    reductions): totals, minima and maxima of each species and of the biomass, the open-voxel count,
    against the same reductions of the oracle's fields."""
    shape = (20, 10, 9)
    nx, ny, nz = shape
    mat = mixed_geometry(*shape, seed=8)
    u = flow_field(oracle, mat, shape)
    N = mat.size
    bio = np.zeros((2, N))
    bio[0, mat == 3] = 30.0
    bio[1, mat == 4] = 20.0
    D, O = pair(clb, oracle, mat, shape, SPECIES, clb.F64, u, law=3, params=[1e-3, 0.1, 0.4, 1e-5], biomass=bio)
    D.ade_step(47)
    O.step(47)
    r = D.reduce()
    inner = np.zeros((nx, ny, nz), bool)
    inner[1:nx - 1] = True
    open_ = inner.ravel() & np.isin(mat, (2, 3, 4))
    assert r["open_voxels"] == open_.sum() and r["nonfinite"] == 0
    for s in range(len(SPECIES)):
        c = O.concentration(s)[open_]
        np.testing.assert_allclose(r["total"][s], c.sum(), rtol=1e-11)
        np.testing.assert_allclose(r["min"][s], c.min(), rtol=1e-11, atol=1e-14)
        np.testing.assert_allclose(r["max"][s], c.max(), rtol=1e-11)
    ob = O.biomass()
    for m in range(2):
        np.testing.assert_allclose(r["biomass"][m], ob[m][inner.ravel()].sum(), rtol=1e-11)
