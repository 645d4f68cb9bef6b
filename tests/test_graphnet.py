"""The oracle's restatement of the graph-network rate laws pinned to the reference's own reader and
evaluator (complab3d_graphnet.hh), whose values are the golden vectors of tests/golden/graphnet.json
(made by tests/golden/make_golden_graphnet.py from the seeded networks of tests/golden/gnn and, in a
checkout of the reference, its example network)."""
import json
import os

import numpy as np
import pytest

HERE = os.path.dirname(__file__)
GOLD = json.load(open(os.path.join(HERE, "golden", "graphnet.json")))
OWN = [c for c in GOLD if not c.get("in_reference_checkout")]
EXAMPLE = [c for c in GOLD if c.get("in_reference_checkout")]


@pytest.mark.parametrize("case", OWN, ids=[c["file"] for c in OWN])
def test_oracle_evaluation_equals_the_reference(oracle, case):
    got = oracle.gnn_eval(os.path.join(HERE, "golden", "gnn", case["file"]), np.array(case["conc"]))
    want = np.array(case["out"])
    assert got.shape == want.shape
    # the same FP64 operations in the same order with the C library's tanh: the same bits
    np.testing.assert_array_equal(got, want)


@pytest.mark.parametrize("case", EXAMPLE, ids=[c["file"] for c in EXAMPLE])
def test_oracle_on_the_reference_example_network(oracle, case):
    """The reference's own trained network (examples/18_graph_network), read from the checkout
    named by CLB_REFERENCE_SRC."""
    ref = os.environ.get("CLB_REFERENCE_SRC", "")
    path = os.path.join(ref, case["file"])
    if not ref or not os.path.isfile(path):
        pytest.skip("CLB_REFERENCE_SRC does not name a checkout of the reference")
    np.testing.assert_array_equal(oracle.gnn_eval(path, np.array(case["conc"])), np.array(case["out"]))


def test_golden_covers_both_readouts_and_the_clamp():
    by = {c["file"]: c for c in OWN}
    assert {"extent_growth.gnn", "species_growth.gnn", "abiotic_extent.gnn", "largest_species.gnn"} <= set(by)
    for c in OWN:
        assert c["clamped_rows"] > 10
        assert np.abs(np.array(c["out"])).max() > 0
    head = open(os.path.join(HERE, "golden", "gnn", "largest_species.gnn")).read()
    assert "width 16" in head and "rounds 4" in head and "readout species" in head
