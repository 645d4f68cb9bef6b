"""Surrogate organisms (.srg networks) on the GPU: the device evaluator against the reference's own
(golden vectors, tests/golden/srg.json), refusals, and the fused transport step with a surrogate
organism and a graph-network organism sharing the substrates, against the FP64 oracle."""
import json
import os

import numpy as np
import pytest

from helpers import mixed_geometry
from test_ade_gpu import flow_field

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(__file__)
SRG = os.path.join(HERE, "golden", "srg")
GNN = os.path.join(HERE, "golden", "gnn")
GOLD = {c["file"]: c for c in json.load(open(os.path.join(HERE, "golden", "srg.json")))}
NAMES = ["A", "B", "C", "D", "E", "F", "G", "H"]
KC = [0.05, 0.1, 0.02, 0.2, 0.1, 0.1, 0.1, 0.1]
VMAX = [10.0, 5.0, 0.0, 0.0, 1.0, 1.0, 1.0, 1.0]


def domain(clb):
    shape = (10, 6, 6)
    mat = np.full(np.prod(shape), 2, np.int8)
    D = clb.Domain(mat, *shape, 0.8, ade_precision=clb.F64, bio_codes=(3,), perm_ratio=(1.0,))
    D.ade_init([dict(omega_pore=1.0, c0=0.1)] * 8)
    D.set_biomass(np.zeros(mat.size))
    return D


@pytest.mark.parametrize("fname", sorted(GOLD))
def test_device_evaluator_equals_the_reference(clb, fname):
    case = GOLD[fname]
    D = domain(clb)
    D.set_surrogate_organism(os.path.join(SRG, fname), NAMES, 0, KC, VMAX, 24.6, 1e-6)
    got, clamped = D.surrogate_eval(0, np.array(case["x"]))
    want = np.array(case["out"])
    # the same operations, unfused, in the same order; CUDA's exp and pow against the C library's
    np.testing.assert_allclose(got, want, rtol=1e-13, atol=1e-12 * np.abs(want).max())
    assert clamped == case["clamped_rows"]


def test_refusals(clb, tmp_path):
    D = domain(clb)
    path = os.path.join(SRG, "uptake_growth.srg")
    with pytest.raises(clb.ClbError, match="input 'A'"):
        D.set_surrogate_organism(path, ["X", "B", "C", "D", "E", "F", "G", "H"], 0, KC, VMAX, 24.6, 0.0)
    with pytest.raises(clb.ClbError, match="belongs to an organism"):
        D.set_surrogate_organism(path, NAMES, -1, KC, VMAX, 24.6, 0.0)
    with pytest.raises(clb.ClbError, match="biomass_molar_mass"):
        D.set_surrogate_organism(path, NAMES, 0, KC, VMAX, 0.0, 0.0)
    text = open(path).read()
    for broken, msg in [(text.replace("trainmax", "# trainmax"), "range it was fitted"),
                        (text.replace("outputs 3", "outputs 4"), "declares outputs 4"),
                        (text.replace("xymin -1", "xymin -1\nmomentum 0.9"), "unknown keyword"),
                        (text[:text.rindex("B 2")], "not a usable surrogate"),
                        (text.replace("layers 2 10 10 3", "layers 2 40 10 3"), "not a usable|truncated|exceeds")]:
        bad = tmp_path / "bad.srg"
        bad.write_text(broken)
        with pytest.raises(clb.ClbError, match=msg):
            D.set_surrogate_organism(str(bad), NAMES, 0, KC, VMAX, 24.6, 0.0)
    with pytest.raises(clb.ClbError, match="no surrogate"):
        D.surrogate_eval(0, np.zeros((1, 2)))
    D.set_surrogate_organism(path, NAMES, 0, KC, VMAX, 24.6, 0.0)
    out, _ = D.surrogate_eval(0, np.full((2, 2), 5.0))
    assert out.shape == (2, 3)
    # a compiled law replaces it
    D.set_kinetics(clb.LAW_DECAY, [1e-3] * 8, 1.0)
    with pytest.raises(clb.ClbError, match="no surrogate"):
        D.surrogate_eval(0, np.zeros((1, 2)))


def test_transport_with_a_surrogate_organism_matches_the_oracle(clb, oracle):
    """A surrogate organism (uptake_growth.srg on microbe 0, biofilm code 3: Michaelis-Menten
    estimates with and without a maximum uptake flux, growth from the network) and a graph-network
    organism (microbe 1, code 4) drawing on the same substrates, FP64 transport over 60 steps of
    30 s, against the oracle to 1e-12."""
    shape = (16, 9, 8)
    mat = mixed_geometry(*shape, seed=16)
    u = flow_field(oracle, mat, shape)
    names = NAMES[:4]
    sp = [dict(omega_pore=1 / 0.9, omega_biofilm=1 / 0.7, left_type=0, right_type=1, left_bc=0.8, c0=0.4),
          dict(omega_pore=1 / 0.8, omega_biofilm=1 / 0.6, left_type=0, right_type=1, left_bc=0.5, c0=0.3),
          dict(omega_pore=1 / 1.1, omega_biofilm=1 / 0.9, left_type=1, right_type=1, c0=0.05),
          dict(omega_pore=1.0, mobile=0, left_type=1, right_type=1, c0=0.02)]
    rng = np.random.default_rng(11)
    bio = np.zeros((2, mat.size))
    bio[0, mat == 3] = rng.uniform(5e-3, 6e-2, (mat == 3).sum())
    bio[1, mat == 4] = rng.uniform(5, 60, (mat == 4).sum())
    kc, vmax = KC[:4], VMAX[:4]
    D = clb.Domain(mat, *shape, 0.8, ade_precision=clb.F64, bio_codes=(3, 4), perm_ratio=(0.3, 0.3))
    D.ade_init(sp)
    D.set_velocity(u)
    D.set_biomass(bio)
    D.set_kinetics(clb.LAW_NONE, [], 30.0)
    D.set_surrogate_organism(os.path.join(SRG, "uptake_growth.srg"), names, 0, kc, vmax, 24.6, 2e-6)
    D.set_graph_network(os.path.join(GNN, "species_growth.gnn"), names, 1)
    O = oracle.OracleAde(mat, *shape, sp, u, bio_codes=(3, 4))
    O.set_biomass(bio)
    O.set_kinetics(0, [], 30.0)
    O.set_surrogate(os.path.join(SRG, "uptake_growth.srg"), names, 0, kc, vmax, 24.6, 2e-6)
    O.set_graph_network(os.path.join(GNN, "species_growth.gnn"), names, 1)
    D.ade_step(60)
    O.step(60)
    for s in range(4):
        np.testing.assert_allclose(D.concentration(s), O.concentration(s), rtol=0, atol=1e-12, err_msg=names[s])
    ob = O.biomass()
    for m in range(2):
        np.testing.assert_allclose(D.biomass(m), ob[m], rtol=1e-12, atol=1e-14)
        assert np.abs(D.biomass(m) - bio[m]).max() > 1e-9
