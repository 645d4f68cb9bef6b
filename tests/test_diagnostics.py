"""The run summary (diagnostics.py) against the reference's own complab_diag::Diagnostics
(complab3d_diagnostics.hh, compiled by tests/golden/make_golden_diag.py into
tests/golden/diagnostics.json): the same rows give the same CSV data lines, the same drift,
negative-value and unknown-substrate messages and the same per-check verdicts. Explanatory prose
(CSV comment lines, advice after a warning) is this library's own and is not compared."""
import json
import os

import numpy as np
import pytest

import diagnostics as dg

CASES = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "diagnostics.json")))
KEY = ("MASS BALANCE", "  [DIAG]   started", "went negative", "names a substrate that", "worst relative drift",
       "[DIAG] verdict: PASS", "[DIAG] verdict: FAIL")


def key_lines(text):
    out = [l for l in text.splitlines() if any(k in l for k in KEY)]
    out += [l[:l.index("NOT CHECKED") + 11] for l in text.splitlines() if "verdict: NOT CHECKED" in l]
    return out


@pytest.mark.parametrize("i", range(len(CASES)))
def test_summary_matches_the_reference(tmp_path, i):
    c = CASES[i]
    path = os.path.join(tmp_path, "summary.csv")
    d = dg.Diagnostics()
    d.configure(True, path, c["tol"])
    for e in c["exprs"]:
        d.add_conserve(e)
    msgs = ""
    stats = np.array(c["stats"])
    for r in range(len(c["iterations"])):
        fields = [dg.FieldStat(n, *stats[r, f]) for f, n in enumerate(c["names"])]
        msgs += d.record(dg.Row(c["iterations"][r], c["porosity"][r], c["open_voxels"][r], fields))
    report = d.final_report().replace(path, "<csv>")
    data = lambda t: [l for l in t.splitlines() if not l.startswith("#")]
    assert data(open(path).read()) == data(c["csv"])
    assert key_lines(msgs) == key_lines(c["messages"])
    assert key_lines(report) == key_lines(c["report"])
    assert d.failed() == ("verdict: FAIL" in c["report"] or "went negative" in c["messages"])
