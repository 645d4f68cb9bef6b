"""The oracle's restatement of the surrogate networks (.srg, complab3d_surrogate.hh) pinned to the
reference's own reader and evaluator (golden vectors of tests/golden/srg.json, made by
tests/golden/make_golden_srg.py) and, in a checkout of the reference, to the reference's own golden
pair tests/parity_net.srg + tests/parity_net_reference.csv."""
import json
import os

import numpy as np
import pytest

HERE = os.path.dirname(__file__)
GOLD = json.load(open(os.path.join(HERE, "golden", "srg.json")))


@pytest.mark.parametrize("case", GOLD, ids=[c["file"] for c in GOLD])
def test_oracle_evaluation_equals_the_reference(oracle, case):
    got = oracle.srg_eval(os.path.join(HERE, "golden", "srg", case["file"]), np.array(case["x"]))
    want = np.array(case["out"])
    assert got.shape == want.shape
    np.testing.assert_array_equal(got, want)


def test_oracle_on_the_reference_golden_pair(oracle):
    """parity_net.srg and its 512 reference predictions (inside the training box), which the
    reference's own test feeds to its evaluator expecting agreement to about 1e-12 relative."""
    ref = os.environ.get("CLB_REFERENCE_SRC", "")
    net = os.path.join(ref, "tests", "parity_net.srg")
    table = os.path.join(ref, "tests", "parity_net_reference.csv")
    if not ref or not os.path.isfile(net):
        pytest.skip("CLB_REFERENCE_SRC does not name a checkout of the reference")
    rows = [r for r in open(table) if r.strip() and not r.startswith("#")]
    data = np.array([[float(v) for v in r.split(",")] for r in rows if r[0].isdigit() or r[0] == "-"])
    X, want = data[:, :2], data[:, 2:]
    got = oracle.srg_eval(net, X)
    assert got.shape == want.shape and len(got) == 512
    np.testing.assert_allclose(got, want, rtol=1e-12, atol=1e-13)


def test_golden_covers_the_cases():
    by = {c["file"]: c for c in GOLD}
    assert set(by) == {"uptake_growth.srg", "log_growth.srg", "positional.srg", "largest.srg"}
    assert by["positional.srg"]["inputs"] is None
    for c in GOLD:
        assert c["clamped_rows"] > 10
    assert (np.array(by["largest.srg"]["out"])[:, 0] == 0).any()  # the growth floor acts
