"""The oracle's biofilm automaton passes against the reference's own: tests/golden/automaton.npz
holds seeded maps whose biomass changes after the automaton's set-up, run through the reference's
updateLocalMaskNtotalLattices3D (one pass) and updateAgeDistance3D (3 sweeps, and to a fixed point
or 1000 sweeps), both from complab3d_processors_part2.hh compiled against oracle/palabos_shim.hh by
tests/golden/make_golden.py. The GPU automaton is checked bit for bit against the oracle in
tests/test_biofilm_ca_gpu.py, so this pins that chain to the reference."""
import os

import numpy as np
import pytest

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "automaton.npz"))
CASES = sorted({int(k.split("_")[0]) for k in GOLD.files if k[0].isdigit()})
SHAPE = tuple(int(v) for v in GOLD["shape"])
BMAX, FRAC = (float(v) for v in GOLD["prm"])


def _case(case):
    return {k.split("_", 1)[1]: GOLD[k] for k in GOLD.files if k.startswith(f"{case}_")}


def _oracle_after_setup(oracle, g):
    N = int(np.prod(SHAPE))
    O = oracle.OracleAde(g["mat"], *SHAPE, [dict(omega_pore=1.0, c0=0.1)], np.zeros(3 * N), bio_codes=(3, 4))
    O.set_biomass(g["bio"])
    O.ca_setup(BMAX, FRAC, 7)
    total0, age0 = O.ca_fields()
    np.testing.assert_array_equal(age0, g["age0"])
    np.testing.assert_array_equal(O.ca_open_flags(), g["flags"])
    np.testing.assert_allclose(total0, g["total0"], rtol=0, atol=1e-12)
    O.set_biomass(g["bio2"])
    return O


@pytest.mark.parametrize("case", CASES)
def test_oracle_mask_and_total_match_the_reference(oracle, case):
    g = _case(case)
    O = _oracle_after_setup(oracle, g)
    O.ca_mask_total_once()
    total, _ = O.ca_fields()
    mask = O.material().astype(np.int32)
    assert (g["mask"] != g["mat"]).sum() > 10  # voxels change code in this case
    np.testing.assert_array_equal(mask, g["mask"])
    np.testing.assert_allclose(total, g["total"], rtol=0, atol=1e-12 * BMAX)


@pytest.mark.parametrize("case", CASES)
def test_oracle_age_relaxation_matches_the_reference(oracle, case):
    g = _case(case)
    O = _oracle_after_setup(oracle, g)
    O.ca_mask_total_once()
    assert O.ca_age_relax(3) == int(g["sweeps"][0])
    np.testing.assert_array_equal(O.ca_fields()[1], g["age3"])
    O2 = _oracle_after_setup(oracle, g)
    O2.ca_mask_total_once()
    assert O2.ca_age_relax(1000) == int(g["sweeps"][1])
    np.testing.assert_array_equal(O2.ca_fields()[1], g["age_fix"])
    assert (g["age3"] != g["age0"]).any()
