"""Graph-network rate laws (.gnn files) on the GPU: the device evaluator against the reference's own
(golden vectors, tests/golden/graphnet.json), refusals, and the fused transport step with two
organisms' networks and an abiotic network against the FP64 oracle."""
import json
import os

import numpy as np
import pytest

from helpers import mixed_geometry
from test_ade_gpu import flow_field

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(__file__)
GNN = os.path.join(HERE, "golden", "gnn")
GOLD = {c["file"]: c for c in json.load(open(os.path.join(HERE, "golden", "graphnet.json")))
        if not c.get("in_reference_checkout")}
NAMES = ["A", "B", "C", "D", "E"]


def domain(clb, n_species=5):
    shape = (10, 6, 6)
    mat = np.full(np.prod(shape), 2, np.int8)
    D = clb.Domain(mat, *shape, 0.8, ade_precision=clb.F64, bio_codes=(3,), perm_ratio=(1.0,))
    D.ade_init([dict(omega_pore=1.0, c0=0.1)] * n_species)
    D.set_biomass(np.zeros(mat.size))
    return D


@pytest.mark.parametrize("fname", sorted(GOLD))
def test_device_evaluator_equals_the_reference(clb, fname):
    case = GOLD[fname]
    D = domain(clb)
    microbe = -1 if not case["growth"] else 0
    D.set_graph_network(os.path.join(GNN, fname), NAMES, microbe)
    got, clamped = D.graph_network_eval(microbe, np.array(case["conc"]))
    # the same operations, unfused, in the same order; CUDA's tanh against the C library's differs by
    # an ulp or two, which the readout's unscaling (a difference of numbers near the output scale)
    # can raise to a few 1e-13 of that scale
    want = np.array(case["out"])
    np.testing.assert_allclose(got, want, rtol=1e-13, atol=1e-12 * np.abs(want).max())
    assert clamped == case["clamped_rows"]


def test_refusals(clb, tmp_path):
    D = domain(clb)
    with pytest.raises(clb.ClbError, match="growth output"):
        D.set_graph_network(os.path.join(GNN, "extent_growth.gnn"), NAMES, -1)
    with pytest.raises(clb.ClbError, match="trained on species 'D'"):
        D.set_graph_network(os.path.join(GNN, "extent_growth.gnn"), ["A", "B", "C", "X", "E"], 0)
    text = open(os.path.join(GNN, "abiotic_extent.gnn")).read()
    for broken, msg in [(text.replace("trainmax", "# trainmax"), "incomplete"),
                        (text.replace("readout extent", "readout sideways"), "readout"),
                        (text.replace("trainmin", "learning_rate 3\ntrainmin"), "unknown keyword"),
                        (text.replace("width 5", "width 17"), "width 17"),
                        (text.replace("species B C D", "species B C"), "names 2 species")]:
        bad = tmp_path / "bad.gnn"
        bad.write_text(broken)
        with pytest.raises(clb.ClbError, match=msg):
            D.set_graph_network(str(bad), NAMES, -1)
    with pytest.raises(clb.ClbError, match="no graph network"):
        D.graph_network_eval(0, np.zeros((1, 4)))
    # a refused file leaves nothing bound; a good one binds
    D.set_graph_network(os.path.join(GNN, "abiotic_extent.gnn"), NAMES, -1)
    out, _ = D.graph_network_eval(-1, np.full((2, 3), 0.5))
    assert out.shape == (2, 3)


def test_transport_with_networks_matches_the_oracle(clb, oracle):
    """Two organisms' networks (an EXTENT readout with growth on microbe 0, biofilm code 3; a
    SPECIES readout with growth on microbe 1, code 4) sharing the substrates' headroom, and an
    abiotic network, in one FP64 transport run, against the oracle to 1e-12."""
    shape = (16, 9, 8)
    mat = mixed_geometry(*shape, seed=15)
    u = flow_field(oracle, mat, shape)
    names = NAMES[:4]
    sp = [dict(omega_pore=1 / 0.9, omega_biofilm=1 / 0.7, left_type=0, right_type=1, left_bc=0.8, c0=0.4),
          dict(omega_pore=1 / 0.8, omega_biofilm=1 / 0.6, left_type=0, right_type=1, left_bc=0.5, c0=0.3),
          dict(omega_pore=1 / 1.1, omega_biofilm=1 / 0.9, left_type=1, right_type=1, c0=0.05),
          dict(omega_pore=1.0, mobile=0, left_type=1, right_type=1, c0=0.0)]
    rng = np.random.default_rng(10)
    bio = np.zeros((2, mat.size))
    bio[0, mat == 3] = rng.uniform(5, 60, (mat == 3).sum())
    bio[1, mat == 4] = rng.uniform(5, 60, (mat == 4).sum())
    D = clb.Domain(mat, *shape, 0.8, ade_precision=clb.F64, bio_codes=(3, 4), perm_ratio=(0.3, 0.3))
    D.ade_init(sp)
    D.set_velocity(u)
    D.set_biomass(bio)
    D.set_kinetics(clb.LAW_NONE, [], 30.0)
    D.set_graph_network(os.path.join(GNN, "extent_growth.gnn"), names, 0)
    D.set_graph_network(os.path.join(GNN, "species_growth.gnn"), names, 1)
    D.set_graph_network(os.path.join(GNN, "abiotic_extent.gnn"), names, -1)
    O = oracle.OracleAde(mat, *shape, sp, u, bio_codes=(3, 4))
    O.set_biomass(bio)
    O.set_kinetics(0, [], 30.0)
    O.set_graph_network(os.path.join(GNN, "extent_growth.gnn"), names, 0)
    O.set_graph_network(os.path.join(GNN, "species_growth.gnn"), names, 1)
    O.set_graph_network(os.path.join(GNN, "abiotic_extent.gnn"), names, -1)
    D.ade_step(60)
    O.step(60)
    for s in range(4):
        np.testing.assert_allclose(D.concentration(s), O.concentration(s), rtol=0, atol=1e-12, err_msg=names[s])
    ob = O.biomass()
    for m in range(2):
        np.testing.assert_allclose(D.biomass(m), ob[m], rtol=1e-12, atol=1e-12)
        assert np.abs(D.biomass(m) - bio[m]).max() > 1e-9  # the organisms grew or decayed
    # the abiotic network acts: without it the oracle's species differ
    O2 = oracle.OracleAde(mat, *shape, sp, u, bio_codes=(3, 4))
    O2.set_biomass(bio)
    O2.set_kinetics(0, [], 30.0)
    O2.set_graph_network(os.path.join(GNN, "extent_growth.gnn"), names, 0)
    O2.set_graph_network(os.path.join(GNN, "species_growth.gnn"), names, 1)
    O2.step(60)
    assert max(np.abs(D.concentration(s) - O2.concentration(s)).max() for s in range(4)) > 1e-9


def test_network_replaces_a_file_law_and_back(clb, oracle):
    """A network bound to a slot replaces the .sym law there and the other way round; a compiled
    law (clb_set_kinetics) replaces both."""
    D = domain(clb, 3)
    sym = os.path.join(HERE, "golden", "sym", "monod_pair.sym")
    D.set_symbolic_kinetics(sym, ["donor", "acceptor", "product"], 0, "cells")
    D.set_graph_network(os.path.join(GNN, "species_growth.gnn"), ["A", "B", "C"], 0)
    with pytest.raises(clb.ClbError, match="no rate-law file"):
        D.symbolic_eval(0, np.zeros((1, 4)))
    D.set_symbolic_kinetics(sym, ["donor", "acceptor", "product"], 0, "cells")
    with pytest.raises(clb.ClbError, match="no graph network"):
        D.graph_network_eval(0, np.zeros((1, 3)))
    D.set_graph_network(os.path.join(GNN, "species_growth.gnn"), ["A", "B", "C"], 0)
    D.set_kinetics(clb.LAW_DECAY, [1e-3] * 3, 1.0)
    with pytest.raises(clb.ClbError, match="no graph network"):
        D.graph_network_eval(0, np.zeros((1, 3)))
