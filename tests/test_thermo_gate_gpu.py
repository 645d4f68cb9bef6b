"""The thermodynamic gate of the biotic rates on the GPU against the FP64 oracle, whose gate is
pinned to the reference's complab3d_thermo.hh (tests/test_kinetics_golden.py)."""
import numpy as np
import pytest

from helpers import mixed_geometry, rel_l2
from test_ade_gpu import SPECIES, flow_field, pair

pytestmark = pytest.mark.gpu

# A -> products with A = species 0, B = species 1 consumed and C = species 2 produced; dG0 chosen so
# that F_T runs from about 1 to 0 across the domain
GATE = dict(species=(0, 1, 2), nu=(-1.0, -1.0, 1.0), dG0=-20.0, atp=0.25, dGatp=50.0, chi=1.0, cmin=1e-9,
            dGloss=0.0, temperature=298.15, gas_constant=8.314462618e-3, conc_scale=1.0)


def gated_pair(clb, oracle, prec, gate=True, seed=4):
    shape = (16, 9, 8)
    mat = mixed_geometry(*shape, seed=seed)
    u = flow_field(oracle, mat, shape)
    rng = np.random.default_rng(2)
    bio = np.zeros((2, mat.size))
    bio[0, mat == 3] = rng.uniform(10, 60, size=(mat == 3).sum())
    bio[1, mat == 4] = rng.uniform(10, 60, size=(mat == 4).sum())
    D, O = pair(clb, oracle, mat, shape, SPECIES, prec, u, law=3, params=[1e-3, 0.1, 0.4, 1e-5], biomass=bio)
    if gate:
        D.set_thermo_gate(**GATE)
        O.set_thermo(**GATE)
    return D, O


def test_f64_gated_dual_monod_matches_oracle(clb, oracle):
    D, O = gated_pair(clb, oracle, clb.F64)
    D.ade_step(80)
    O.step(80)
    for s in range(3):
        np.testing.assert_allclose(D.concentration(s), O.concentration(s), rtol=0, atol=1e-12)
    ob = O.biomass()
    for m in range(2):
        np.testing.assert_allclose(D.biomass(m), ob[m], rtol=1e-12, atol=1e-12)
    # the gate acts: the ungated run differs
    _, U = gated_pair(clb, oracle, clb.F64, gate=False)
    U.step(80)
    assert np.max(np.abs(U.biomass()[0] - ob[0])) > 1e-6


@pytest.mark.parametrize("prec,tol", [("F32", 1e-5), ("F16S", 3e-2)])
def test_reduced_precision_gated_dual_monod_error(clb, oracle, prec, tol):
    D, O = gated_pair(clb, oracle, getattr(clb, prec))
    D.ade_step(80)
    O.step(80)
    for s in range(3):
        assert rel_l2(D.concentration(s), O.concentration(s)) < tol, s
    ob = O.biomass()
    for m in range(2):
        assert rel_l2(D.biomass(m), ob[m]) < tol, m


def test_gate_without_microbes_changes_nothing(clb, oracle):
    """The block applies to microbe 0, so a run without biomass fields is not gated."""
    shape = (14, 8, 9)
    mat = mixed_geometry(*shape, seed=6)
    u = flow_field(oracle, mat, shape)
    runs = []
    for gate in (False, True):
        D, _ = pair(clb, oracle, mat, shape, SPECIES, clb.F64, u, law=1, params=[1e-3, 2e-2, 5e-3])
        if gate:
            D.set_thermo_gate(**GATE)
        D.ade_step(30)
        runs.append([D.concentration(s) for s in range(3)])
        D.close()
    for a, b in zip(*runs):
        np.testing.assert_array_equal(a, b)


def test_gate_off_again_restores_the_ungated_step(clb, oracle):
    D, _ = gated_pair(clb, oracle, clb.F64)
    D.set_thermo_gate()  # no terms: off
    D.ade_step(20)
    E, _ = gated_pair(clb, oracle, clb.F64, gate=False)
    E.ade_step(20)
    for s in range(3):
        np.testing.assert_array_equal(D.concentration(s), E.concentration(s))


@pytest.mark.parametrize("bad", [dict(cmin=0.0), dict(dGloss=-1.0), dict(temperature=0.0), dict(species=(0, 1, 9))])
def test_gate_rejects_bad_blocks(clb, oracle, bad):
    D, _ = gated_pair(clb, oracle, clb.F64, gate=False)
    g = dict(GATE, **bad)
    with pytest.raises(clb.ClbError):
        D.set_thermo_gate(**g)


def test_batch_refuses_a_gated_domain(clb, oracle):
    """The batched transport kernels are compiled without the gate, so a gated domain is refused."""
    D, _ = gated_pair(clb, oracle, clb.F64)
    with pytest.raises(clb.ClbError):
        clb.Batch([D])


def test_fp32_gate_keeps_relative_precision_near_the_threshold(clb, oracle):
    """With x = (dG + m dG_ATP)/(chi R T) in [-1e-3, 0) the gate is F_T = -expm1(x) ~ |x|. The FP32
    lattice evaluates it to the FP64 lattice's value within 1e-4 relative per voxel: the constant
    part of x is formed in FP64 (no cancellation of dG0 against m dG_ATP in FP32) and F_T comes
    from expm1 (no cancellation of 1 - exp(x)). Compared on one step's biomass increment (decay
    off), which is the gated growth rate itself."""
    shape = (16, 9, 8)
    mat = mixed_geometry(*shape, seed=4)
    u = flow_field(oracle, mat, shape)
    rng = np.random.default_rng(7)
    bio = np.zeros((2, mat.size))
    bio[0, mat == 3] = rng.uniform(10, 60, size=(mat == 3).sum())
    bio[1, mat == 4] = rng.uniform(10, 60, size=(mat == 4).sum())
    RT = 8.314462618e-3 * 298.15
    incs = {}
    for xs in (-1e-4, -7e-4):
        # a tiny stoichiometric number keeps ln Q's part of x (|nu ln a| <= 1e-8 x 20.8) below
        # 1 % of it; the donor starts at 0.5 everywhere so every biofilm voxel grows in the first step
        gate = dict(GATE, species=(0,), nu=(1e-8,), atp=0.25, dGatp=50.0, dG0=-12.5 + xs * RT)
        species = [dict(SPECIES[0], c0=0.5)] + SPECIES[1:]
        for prec in (clb.F64, clb.F32):
            D, _ = pair(clb, oracle, mat, shape, species, prec, u, law=3, params=[1e-3, 0.1, 0.4, 0.0],
                        biomass=bio)
            D.set_thermo_gate(**gate)
            D.ade_step(1)
            incs[prec] = D.biomass(0) - bio[0]
            D.close()
        live = incs[clb.F64] > 0
        assert live.sum() > 10
        ratio = incs[clb.F64][live] / (-np.expm1(xs))
        assert np.all(ratio > 0)
        err = np.abs(incs[clb.F32][live] / incs[clb.F64][live] - 1.0)
        assert err.max() < 1e-4, (xs, err.max())
