"""Run-time rate laws (.sym files) on the GPU: the device interpreter against the reference's own
evaluator (golden vectors, tests/golden/symbolic.json), and the fused transport step with an
organism's law and an abiotic law against the FP64 oracle."""
import json
import os

import numpy as np
import pytest

from helpers import mixed_geometry
from test_ade_gpu import flow_field

pytestmark = pytest.mark.gpu
GOLD = {c["file"]: c for c in json.load(open(os.path.join(os.path.dirname(__file__), "golden", "symbolic.json")))}
SYM = os.path.join(os.path.dirname(__file__), "golden", "sym")

# species the files bind to, and the organism's biomass variable
BINDINGS = {
    "monod_pair.sym": (["donor", "acceptor", "product"], 0, "cells"),
    "derived_hourly.sym": (["acetate", "o2", "co2"], 0, "Bug"),
    "extent_abiotic.sym": (["Fe", "HS", "FeS"], -1, ""),
    "functions.sym": (["a", "b", "c", "p", "q", "r", "s"], 0, ""),
}


def domain(clb, names, prec=None, bio=True):
    shape = (10, 6, 6)
    mat = np.full(np.prod(shape), 2, np.int8)
    D = clb.Domain(mat, *shape, 0.8, ade_precision=clb.F64 if prec is None else prec, bio_codes=(3,), perm_ratio=(1.0,))
    D.ade_init([dict(omega_pore=1.0, c0=0.1)] * len(names))
    if bio:
        D.set_biomass(np.zeros(mat.size))
    return D


@pytest.mark.parametrize("fname", sorted(BINDINGS))
def test_device_interpreter_equals_the_reference(clb, fname):
    names, microbe, mname = BINDINGS[fname]
    D = domain(clb, names)
    D.set_symbolic_kinetics(os.path.join(SYM, fname), names, microbe, mname)
    case = GOLD[fname]
    got = D.symbolic_eval(microbe, np.array(case["vars"]))
    # CUDA's exp / log / pow / tanh against the C library's: a few ulp
    np.testing.assert_allclose(got, np.array(case["rates_out"]), rtol=1e-13, atol=1e-300)


def test_refusals(clb, tmp_path):
    names = ["donor", "acceptor", "product"]
    D = domain(clb, names)
    with pytest.raises(clb.ClbError, match="extent"):
        D.set_symbolic_kinetics(os.path.join(SYM, "extent_abiotic.sym"), ["Fe", "HS", "FeS"], 0, "x")
    with pytest.raises(clb.ClbError, match="neither a substrate"):
        D.set_symbolic_kinetics(os.path.join(SYM, "monod_pair.sym"), names, 0, "biomass")
    bad = tmp_path / "bad.sym"
    bad.write_text("vars a b\nrate growth = a * (b + 1\n")
    with pytest.raises(clb.ClbError, match="missing"):
        D.set_symbolic_kinetics(str(bad), ["a", "b", "c"], 0, "")
    # a refused file leaves no law behind; with one installed the batch refuses the domain (the
    # batched kernels carry no rate-law interpreter)
    D.set_symbolic_kinetics(os.path.join(SYM, "monod_pair.sym"), names, 0, "cells")
    with pytest.raises(clb.ClbError):
        clb.Batch([D])


def test_transport_with_file_laws_matches_the_oracle(clb, oracle):
    """An organism's law (monod_pair.sym on microbe 0, biofilm code 3) and an abiotic law
    (extent_abiotic.sym) in one FP64 transport run, against the oracle to 1e-12."""
    shape = (16, 9, 8)
    mat = mixed_geometry(*shape, seed=14)
    u = flow_field(oracle, mat, shape)
    names = ["donor", "acceptor", "product", "Fe", "HS", "FeS"]
    sp = [dict(omega_pore=1 / 0.9, omega_biofilm=1 / 0.7, left_type=0, right_type=1, left_bc=0.8, c0=0.3),
          dict(omega_pore=1 / 0.8, omega_biofilm=1 / 0.6, left_type=0, right_type=1, left_bc=0.5, c0=0.2),
          dict(omega_pore=1 / 1.1, omega_biofilm=1 / 0.9, left_type=1, right_type=1, c0=0.0),
          dict(omega_pore=1 / 0.9, omega_biofilm=1 / 0.8, left_type=0, right_type=1, left_bc=2e-3, c0=1e-3),
          dict(omega_pore=1 / 0.9, omega_biofilm=1 / 0.8, left_type=0, right_type=1, left_bc=3e-3, c0=1e-3),
          dict(omega_pore=1.0, mobile=0, left_type=1, right_type=1, c0=0.0)]
    rng = np.random.default_rng(9)
    bio = np.zeros((2, mat.size))
    bio[0, mat == 3] = rng.uniform(5, 60, (mat == 3).sum())
    bio[1, mat == 4] = rng.uniform(5, 60, (mat == 4).sum())
    D = clb.Domain(mat, *shape, 0.8, ade_precision=clb.F64, bio_codes=(3, 4), perm_ratio=(0.3, 0.3))
    D.ade_init(sp)
    D.set_velocity(u)
    D.set_biomass(bio)
    D.set_kinetics(clb.LAW_NONE, [], 2.0)  # the time step the file's rates (per second) apply over
    D.set_symbolic_kinetics(os.path.join(SYM, "monod_pair.sym"), names, 0, "cells")
    D.set_symbolic_kinetics(os.path.join(SYM, "extent_abiotic.sym"), names, -1, "")
    O = oracle.OracleAde(mat, *shape, sp, u, bio_codes=(3, 4))
    O.set_biomass(bio)
    O.set_kinetics(0, [], 2.0)
    O.set_symbolic(os.path.join(SYM, "monod_pair.sym"), names, 0, "cells")
    O.set_symbolic(os.path.join(SYM, "extent_abiotic.sym"), names, -1, "")
    D.ade_step(60)
    O.step(60)
    for s in range(6):
        np.testing.assert_allclose(D.concentration(s), O.concentration(s), rtol=0, atol=1e-12, err_msg=names[s])
    ob = O.biomass()
    np.testing.assert_allclose(D.biomass(0), ob[0], rtol=1e-12, atol=1e-12)
    assert D.concentration(5).max() > 1e-6        # the abiotic law precipitated FeS
    assert np.abs(D.biomass(0) - bio[0]).max() > 1e-6  # the organism grew
