"""The run summary filled from a domain's reductions: in a closed box without reactions the
conserved sum (total + held = the lattice's whole content) passes at round-off; with decay it
drifts and the check fails; the CSV has one data line per recorded row."""
import os

import numpy as np
import pytest

import diagnostics as dg
from helpers import mixed_geometry
from test_ade_gpu import flow_field, pair

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("decay,verdict", [(0.0, "PASS"), (1e-3, "FAIL")])
def test_summary_of_a_closed_box(clb, oracle, tmp_path, decay, verdict):
    shape = (18, 10, 9)
    mat = mixed_geometry(*shape)
    u = flow_field(oracle, mat, shape)
    sp = [dict(omega_pore=1 / 0.9, omega_biofilm=1 / 0.7, left_type=2, right_type=2, c0=0.3)]
    D, _ = pair(clb, oracle, mat, shape, sp, clb.F64, u, law=1 if decay else 0, params=[decay])
    path = os.path.join(tmp_path, "summary.csv")
    d = dg.Diagnostics()
    d.configure(True, path, 1e-11)
    d.add_conserve("A")
    for it in range(4):
        if it:
            D.ade_step(100)
        row = dg.row_from_domain(D, 100 * it, ["A"])
        assert row.open_voxels > 0 and 0 < row.porosity < 1
        np.testing.assert_allclose(row.fields[0].total, D.reduce()["total"][0])
        d.record(row)
    rep = d.final_report()
    assert ("verdict: " + verdict) in rep
    lines = [l for l in open(path).read().splitlines() if not l.startswith("#")]
    assert lines[0].startswith("iteration,porosity,open_voxels,A_total,A_mean,A_min,A_max,A_held")
    assert len(lines) == 5
