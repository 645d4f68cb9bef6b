"""The oracle's kinetics passes against the reference's own: tests/golden/kinetics.npz holds seeded
fields run through the reference's run_kinetics (complab3d_processors_part1.hh, with the library's
decay / Monod / dual-Monod laws as the rate hook) and through run_abiotic_kinetics and
surfaceAbioticKinetics3D (precipitationVOP.hh) with the reference's FeS precipitation law of
examples/15, compiled against oracle/palabos_shim.hh by tests/golden/make_golden.py.

The reference applies R dt as it is; the method adds one rule, the clamp dC = max(R dt, -C), so a
voxel never goes below zero. Where the reference's increment stays at or above -C the oracle must
equal it (to round-off); where it overdraws, the oracle's increment must be exactly -C. The GPU's
kinetics is checked against the oracle in tests/test_ade_gpu.py, so this pins that chain."""
import os

import numpy as np
import pytest

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "kinetics.npz"))
SHAPE = tuple(int(v) for v in GOLD["shape"])
N = int(np.prod(SHAPE))
THRD = 1e-12  # the reference's threshold: concentrations below it read as zero


def _case(tag):
    return {k.split("_", 1)[1]: GOLD[k] for k in GOLD.files if k.startswith(f"{tag}_")}


def _tags(prefix):
    return sorted({k.split("_")[0] for k in GOLD.files if k.startswith(prefix) and k[1].isdigit()})


def _check(out, ref, conc, tol):
    base = np.where(conc < THRD, 0.0, conc)
    over = ref < -base  # the reference's increment overdraws the voxel
    free = ~over
    np.testing.assert_allclose(out[free], ref[free], rtol=0, atol=tol)
    np.testing.assert_array_equal(out[over], -base[over])
    return int(over.sum())


@pytest.mark.parametrize("tag", _tags("b"))
def test_oracle_biotic_kinetics_matches_the_reference(oracle, tag):
    g = _case(tag)
    law, M, dt = int(g["meta"][0]), int(g["meta"][1]), float(g["meta"][2])
    S = g["C"].shape[0]
    O = oracle.OracleAde(g["mat"], *SHAPE, [dict(omega_pore=1.0)] * S, np.zeros(3 * N), bio_codes=(3,))
    O.set_kinetics(law, g["prm"], dt)
    B = g["B"].reshape(M, N)
    O.set_biomass(B)
    dC, dB = O.biotic_increments(g["C"], B)
    assert np.count_nonzero(g["dC"]) > 500
    _check(dC, g["dC"], g["C"], 1e-14)
    if M:
        _check(dB, g["dB"], B, 1e-14)


@pytest.mark.parametrize("tag", _tags("a"))
def test_oracle_abiotic_kinetics_matches_the_reference(oracle, tag):
    g = _case(tag)
    surf, dt = int(g["meta"][0]), float(g["meta"][1])
    S = g["C"].shape[0]
    O = oracle.OracleAde(g["mat"], *SHAPE, [dict(omega_pore=1.0)] * S, np.zeros(3 * N))
    O.set_abiotic(4, np.array([1.0, 0, 1, 3], np.float64), surf)  # kp = 1, Fe2 + HS -> FeS (examples/15)
    O.set_kinetics(0, np.zeros(1), dt)
    dC = O.abiotic_increments(g["C"])
    assert np.count_nonzero(g["dC"]) > 500
    _check(dC, g["dC"], g["C"], 1e-14)


def test_some_cases_overdraw():
    """The fixture exercises the clamp: some reference increments go below -C."""
    n = 0
    for tag in _tags("b") + _tags("a"):
        g = _case(tag)
        n += int((g["dC"] < -np.where(g["C"] < THRD, 0.0, g["C"])).sum())
    assert n > 100


@pytest.mark.parametrize("tag", _tags("g"))
def test_oracle_thermodynamic_gate_matches_the_reference(oracle, tag):
    """complab3d_thermo.hh's factor F_T = max(0, 1 - exp((dG + m dG_ATP) / (chi R T))) on seeded
    concentration vectors (equal: both evaluate the same expression with the C library's log and
    exp), and run_kinetics gated by it (dual Monod, one microbe)."""
    g = _case(tag)
    S = g["C"].shape[0]
    O = oracle.OracleAde(g["mat"], *SHAPE, [dict(omega_pore=1.0)] * S, np.zeros(3 * N), bio_codes=(3,))
    O.set_thermo(g["sp"], g["nu"], *g["v"])
    F = np.array([O.thermo_factor(c) for c in g["cs"]])
    assert (g["F"] == 0).sum() > 20 and ((g["F"] > 0) & (g["F"] < 1)).sum() > 100
    np.testing.assert_allclose(F, g["F"], rtol=1e-14, atol=1e-15)
    O.set_kinetics(3, g["prm"], 1.0)
    O.set_biomass(g["B"])
    dC, dB = O.biotic_increments(g["C"], g["B"])
    _check(dC, g["dC"], g["C"], 1e-14)
    _check(dB, g["dB"], g["B"], 1e-13)
    O.set_thermo()  # off: the increments change
    dC0, _ = O.biotic_increments(g["C"], g["B"])
    assert (np.abs(dC0 - dC) > 1e-12).sum() > 100
