"""The reference's straight-duct check on the GPU (ABC_sweep_package/tools/analytic_channel.py).

A + B -> C at one diffusivity with every x face held: A - B, A + C and B + C are conservative
tracers. Two statements are exact and checked to round-off: (1) at every step each combination
equals an unreacting species fed with its boundary values (the reaction cancels in the linear
transport), (2) at Pe = 0 its steady cross-section mean is the straight line of the reference's
ade_1d (golden vectors from that function, tests/golden/channel.json). At Pe > 0 the reference
only reports the distance to the 1-D exponential profile (its default tolerance is 2 %); with the
plug flow used here the distance is the lattice's discretisation error (1e-6 at Pe 0.5, 1.3e-4 at
Pe 2 in the oracle), asserted below 1e-3 and printed."""
import numpy as np
import pytest

import channel_case as cc

pytestmark = pytest.mark.gpu


def run(clb, pe, steps, prec):
    D = clb.Domain(cc.material(), cc.NX, cc.NY, cc.NZ, 0.8, ade_precision=prec)
    D.ade_init(cc.species())
    D.set_velocity(cc.velocity(pe))
    D.set_abiotic_kinetics(clb.LAW_PRECIP, cc.ABIOTIC, 0)
    return D


def test_combinations_equal_unreacting_tracers_at_every_step(clb):
    D = run(clb, 0.5, 0, clb.F64)
    for steps in (1, 40, 400, 2000):
        D.ade_step(steps)
        c = [D.concentration(s) for s in range(6)]
        got = cc.combinations(c)
        for k, name in enumerate(("A - B", "A + C", "B + C")):
            np.testing.assert_allclose(got[name], c[3 + k], rtol=0, atol=1e-13, err_msg=name)
    assert np.max(c[2]) > 1e-3  # the reaction is running once A and B meet


def test_pe0_steady_profiles_are_the_reference_straight_lines(clb):
    D = run(clb, 0.0, 0, clb.F64)
    D.ade_step(16000)
    c = [D.concentration(s) for s in range(6)]
    for name, field in cc.combinations(c).items():
        got = cc.cross_section_mean(field)
        want = cc.golden(0.0, name)
        err = np.max(np.abs(got - want))
        print(f"Pe 0 {name}: max |mean - ade_1d| = {err:.2e}")
        assert err < 1e-11, name
    # the reaction sheet sits at the middle for equal feeds and no flow (the checker's thin-sheet
    # prediction 0.5)
    peak = np.argmax(cc.cross_section_mean(c[2]))
    assert abs(peak / (cc.NX - 1) - 0.5) < 0.05


@pytest.mark.parametrize("pe", [0.5, 2.0])
def test_pe_positive_profiles_near_the_reference_exponential(clb, pe):
    D = run(clb, pe, 0, clb.F64)
    D.ade_step(16000)
    c = [D.concentration(s) for s in range(6)]
    for name, field in cc.combinations(c).items():
        got = cc.cross_section_mean(field)
        want = cc.golden(pe, name)
        rel = np.max(np.abs(got - want)) / max(abs(want[0]), abs(want[-1]))
        print(f"Pe {pe} {name}: relative distance to ade_1d {rel:.2e}")
        assert rel < 1e-3, name


@pytest.mark.parametrize("prec,tol", [("F32", 1e-4), ("F16S", 0.1)])
def test_reduced_precision_steady_profile(clb, prec, tol):
    """The FP32 / FP16 lattices against the same straight lines: the storage error of a steady
    state reached through 16000 rounded steps (measured on a B200: FP32 4.3e-5; FP16 1.7e-2 on
    A - B and 6.0e-2 on A + C, where the product's small concentrations enter). FP16 keeps 11
    significant bits, and near a steady state each step's change is below the spacing of the
    stored values, so the rounding does not average out."""
    D = run(clb, 0.0, 0, getattr(clb, prec))
    D.ade_step(16000)
    c = [D.concentration(s) for s in range(6)]
    for name, field in cc.combinations(c).items():
        err = np.max(np.abs(cc.cross_section_mean(field) - cc.golden(0.0, name)))
        print(f"{prec} Pe 0 {name}: {err:.2e}")
        assert err < tol, name
