"""The oracle's dissolution passes against the reference's own: tests/golden/dissolution.npz holds
seeded fields run through the reference's surfaceDissolutionKinetics3D and dissolutionGather3D
(dissolutionVOP.hh, compiled from the reference sources against oracle/palabos_shim.hh by
tests/golden/make_golden.py). Both dissolution laws, with and without the surface-only rule,
negative water and pending increments. The GPU's dissolution is checked against the oracle in
tests/test_geometry_update_gpu.py, so this pins that chain to the reference."""
import os

import numpy as np
import pytest

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "dissolution.npz"))
CASES = sorted({int(k.split("_")[0]) for k in GOLD.files if k[0].isdigit()})


@pytest.mark.parametrize("case", CASES)
def test_oracle_dissolution_matches_the_reference(oracle, case):
    g = {k.split("_", 1)[1]: GOLD[k] for k in GOLD.files if k.startswith(f"{case}_")}
    law, surf, dt, S, sM = g["meta"]
    shape = tuple(int(v) for v in GOLD["shape"])
    out = oracle.dissolution_increments(shape, int(S), int(sM), float(dt), int(law), g["prm"], int(surf), g["mat"],
                                        0, 1, g["stamp"], g["C"], g["dC0"])
    moved = np.abs(g["dC"] - g["dC0"]).max()
    assert moved > 1e-3  # the case dissolves something
    np.testing.assert_allclose(out, g["dC"], rtol=0, atol=1e-13 * max(1.0, np.abs(g["dC"]).max()))
