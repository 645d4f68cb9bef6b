"""The oracle's restatement of the run-time rate-law language pinned to the reference's own reader
and evaluator (complab3d_symbolic.hh), whose values are the golden vectors of
tests/golden/symbolic.json (made by tests/golden/make_golden_symbolic.py)."""
import json
import os

import numpy as np
import pytest

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "symbolic.json")))
SYM = os.path.join(os.path.dirname(__file__), "golden", "sym")


@pytest.mark.parametrize("case", GOLD, ids=[c["file"] for c in GOLD])
def test_oracle_evaluation_equals_the_reference(oracle, case):
    X = np.array(case["vars"])
    want = np.array(case["rates_out"])
    got = oracle.sym_eval(os.path.join(SYM, case["file"]), X)
    assert got.shape == want.shape
    np.testing.assert_allclose(got, want, rtol=1e-15, atol=1e-300)


def test_golden_covers_the_guards():
    """The fixtures exercise the range clamp, the derived lines and the guarded operations."""
    by = {c["file"]: c for c in GOLD}
    assert by["functions.sym"]["clamped_rows"] > 10 and by["monod_pair.sym"]["clamped_rows"] > 5
    assert by["derived_hourly.sym"]["rates"] == ["growth", "acetate", "o2", "co2"]
    assert by["extent_abiotic.sym"]["rates"] == ["extent", "Fe", "HS", "FeS"]
