"""The oracle's node conversions against the reference's own: tests/golden/conversion.npz holds
seeded maps run through the reference's precipNodeConversion3D (precipitationVOP.hh) and, with
dissolution on, dissolNodeConversion3D (dissolutionVOP.hh), compiled against
oracle/palabos_shim.hh by tests/golden/make_golden.py. The GPU's conversions are checked bit for
bit against the oracle in tests/test_geometry_update_gpu.py, so this pins that chain.

The material maps must be equal. The phase (stamp) field is compared with dissolution on: with it
off the reference declares no precipitate phase and stamps nothing, while the oracle (like the
library, which also marks sealed voxels for the flow's permeability ratio) stamps every voxel it
seals; the phase is read only by the dissolution pass, so the maps agree either way."""
import os

import numpy as np
import pytest

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "conversion.npz"))
CASES = sorted({int(k.split("_")[0]) for k in GOLD.files if k[0].isdigit()})
SHAPE = tuple(int(v) for v in GOLD["shape"])
N = int(np.prod(SHAPE))


@pytest.mark.parametrize("case", CASES)
def test_oracle_node_conversion_matches_the_reference(oracle, case):
    g = {k.split("_", 1)[1]: GOLD[k] for k in GOLD.files if k.startswith(f"{case}_")}
    S, sM, full, reopen = GOLD["prm"]
    S, sM = int(S), int(sM)
    pcode, dis = (int(v) for v in g["meta"])
    species = [dict(omega_pore=1.0)] * S
    species[sM] = dict(omega_pore=1.0, mobile=0)
    O = oracle.OracleAde(g["mat"], *SHAPE, species, np.zeros(3 * N), bio_codes=(3,))
    O.set_precip(sM, float(full), precip_code=pcode, dissolution=dis, reopen=float(reopen), pore_code=2)
    O.set_immobile(sM, g["C"][sM])
    O.set_stamp(g["stamp"])
    sealed, reopened = O.geometry_update()
    assert sealed > 10
    if dis and pcode == 0:
        assert reopened > 5
    np.testing.assert_array_equal(O.material(), g["mat_out"])
    # a voxel that already carries the precipitate code counts as sealed again without changing
    assert (O.material() != g["mat"]).sum() <= sealed + reopened
    if dis:
        np.testing.assert_array_equal(O.stamp(), g["stamp_out"])
