"""Biofilm cellular automaton on the GPU against the sequential oracle: bit-exact.

The oracle runs pushExcessBiomass3D / updateLocalMaskNtotalLattices3D / updateAgeDistance3D in the
reference's lexicographic order with the seeded neighbour draws; the GPU runs the parallel
schedule. Biomass, total biomass, mask and age must agree exactly after every iteration."""
import numpy as np
import pytest

from helpers import mixed_geometry

pytestmark = pytest.mark.gpu

BIO = dict(bio_codes=(3, 4), perm_ratio=(0.3, 0.3))
SP = [dict(omega_pore=1 / 0.9, omega_biofilm=1 / 0.7, left_type=0, right_type=1, left_bc=1.0, c0=0.2),
      dict(omega_pore=1 / 0.75, omega_biofilm=1 / 0.6, left_type=1, right_type=1, c0=0.5)]


def setup(clb, oracle, shape, seed, lo, hi, bmax=100.0, frac=0.1, ca_seed=77, half=False):
    mat = mixed_geometry(*shape, seed=seed)
    N = mat.size
    P = shape[1] * shape[2]
    rng = np.random.default_rng(seed)
    bio = np.zeros((2, N))
    bio[0, mat == 3] = rng.uniform(lo, hi, (mat == 3).sum())
    bio[1, mat == 4] = rng.uniform(lo, hi, (mat == 4).sum())
    both = (mat == 3) & (rng.random(N) < 0.5)          # some voxels hold both microbes
    bio[1, both] = rng.uniform(0.2 * lo, 0.5 * hi, both.sum())
    bio[:, :P] = 0.0                                     # ghost planes hold no biomass
    bio[:, -P:] = 0.0
    D = clb.Domain(mat, *shape, 0.8, ade_precision=clb.F64, **BIO)
    D.ade_init(SP)
    D.set_biomass(bio)
    O = oracle.OracleAde(mat, *shape, SP, np.zeros(3 * N), bio_codes=(3, 4))
    O.set_biomass(bio)
    D.ca_setup(bmax, frac, ca_seed, half=half)
    O.ca_setup(bmax, frac, ca_seed, half=half)
    return D, O, mat


def assert_same(D, O):
    ob = O.biomass()
    for m in range(2):
        np.testing.assert_array_equal(D.biomass(m), ob[m], err_msg=f"biomass {m}")
    np.testing.assert_array_equal(D.material(), O.material())
    t, a = O.ca_fields()
    np.testing.assert_array_equal(D.ca_total(), t)
    np.testing.assert_array_equal(D.ca_age(), a)


@pytest.mark.parametrize("shape,seed", [((18, 12, 10), 31), ((24, 16, 13), 32)])
def test_ca_bit_exact_over_growth_cycles(clb, oracle, shape, seed):
    D, O, mat = setup(clb, oracle, shape, seed, 60.0, 420.0)
    swept = 0
    for cycle in range(4):
        st, sw, ch = D.ca_step()
        rc, sw_o, ch_o = O.ca_step()
        assert rc == 0 and (sw, ch) == (sw_o, ch_o), (cycle, sw, ch, sw_o, ch_o)
        swept += sw
        assert_same(D, O)
        # growth between iterations: the same field on both sides
        grown = np.stack([D.biomass(m) for m in range(2)]) * 1.25
        D.set_biomass(grown)
        O.set_biomass(grown)
    assert swept > 1


def test_ca_conserves_biomass(clb, oracle):
    D, O, mat = setup(clb, oracle, (20, 14, 12), 33, 80.0, 500.0)
    before = sum(D.biomass(m).sum() for m in range(2))
    st, sw, ch = D.ca_step()
    after = sum(D.biomass(m).sum() for m in range(2))
    assert sw > 0 and ch
    assert abs(after - before) <= 1e-12 * before
    t = D.ca_total()
    open_ = (D.material() != 0) & (D.material() != 1)
    assert t[open_].max() <= 100.0 + 1e-9


def test_ca_dynamics_refresh_then_transport_matches(clb, oracle):
    """After the mask moves, updateSoluteDynamics3D switches the relaxation rates; transport after
    the refresh matches the oracle to FP64 round-off."""
    shape = (18, 12, 10)
    D, O, mat = setup(clb, oracle, shape, 34, 60.0, 420.0)
    D.ca_step()
    O.ca_step()
    assert (D.material() != mat).any()
    D.refresh_dynamics(species=True, flow=False)
    O.refresh_dynamics()
    rng = np.random.default_rng(5)
    u = np.zeros((3, D.N))
    u[0] = rng.uniform(0, 0.02, D.N)
    D.set_velocity(u)
    O.set_velocity(u)
    D.ade_step(40)
    O.step(40)
    for s in range(2):
        np.testing.assert_allclose(D.ade_populations(s), O.populations(s), rtol=0, atol=1e-12)


def test_ca_then_flow_refresh_runs(clb, oracle):
    """updateNsLatticesDynamics3D on the flow lattice after the automaton: the flow steps on and
    the velocity vanishes in impermeable biofilm."""
    shape = (18, 12, 10)
    mat = mixed_geometry(*shape, seed=35)
    N = mat.size
    P = shape[1] * shape[2]
    bio = np.zeros((2, N))
    bio[0, mat == 3] = 300.0
    bio[1, mat == 4] = 250.0
    bio[:, :P] = 0
    bio[:, -P:] = 0
    D = clb.Domain(mat, *shape, 0.8, flow_precision=clb.F64, ade_precision=clb.F64, bio_codes=(3, 4),
                   perm_ratio=(0.0, 0.0))
    D.flow_init(1e-4)
    D.flow_step(100)
    D.ade_init(SP)
    D.set_biomass(bio)
    D.ca_setup(100.0, 0.1, 5)
    st, sw, ch = D.ca_step()
    assert ch
    D.refresh_dynamics(species=True, flow=True)
    D.flow_step(200)
    u = D.velocity()
    assert np.isfinite(u).all()
    m = D.material()
    biofilm = (m != 0) & (m != 1) & (m != 2)
    assert np.abs(u[:, biofilm]).max() == 0.0
    assert np.abs(u[0, m == 2]).max() > 0.0


@pytest.mark.parametrize("shape,seed", [((18, 12, 10), 41), ((24, 16, 13), 42)])
def test_ca_half_push_bit_exact_over_growth_cycles(clb, oracle, shape, seed):
    """'half' push mode (halfPushExcessBiomass3D, complab3d_processors_part1.hh:735-970): biofilm
    voxels above the maximum push half their biomass; the GPU equals the sequential oracle bit for
    bit after every iteration, and the total biomass is conserved to round-off."""
    D, O, mat = setup(clb, oracle, shape, seed, 60.0, 420.0, half=True)
    swept = 0
    for cycle in range(4):
        before = sum(D.biomass(m).sum() for m in range(2))
        st, sw, ch = D.ca_step()
        rc, sw_o, ch_o = O.ca_step()
        assert rc == 0 and (sw, ch) == (sw_o, ch_o), (cycle, sw, ch, sw_o, ch_o)
        swept += sw
        assert_same(D, O)
        after = sum(D.biomass(m).sum() for m in range(2))
        assert abs(after - before) <= 1e-12 * before
        grown = np.stack([D.biomass(m) for m in range(2)]) * 1.25
        D.set_biomass(grown)
        O.set_biomass(grown)
    assert swept > 1


def test_half_and_fraction_differ(clb, oracle):
    """The two push modes are different automata on the same state."""
    runs = []
    for half in (False, True):
        D, O, mat = setup(clb, oracle, (18, 12, 10), 43, 60.0, 420.0, half=half)
        D.ca_step()
        runs.append(np.stack([D.biomass(m) for m in range(2)]))
    assert np.max(np.abs(runs[0] - runs[1])) > 1.0
