"""The CompLaB.xml reader (clb_case_*) on CPU: parameters, defaults, the reference's error cases,
and the unit chain of complab.cpp:1213-1253 where it needs no flow solve (Pe = 0), restated here."""
import glob
import os

import numpy as np
import pytest

import case_files


def unit_chain(tau, dx, d_pore, d_bio):
    """complab.cpp:1221-1253 at Pe = 0: refTau = tau, refNu = cs2 (refTau - 1/2) with cs2 = 1/4,
    ade_dt = refNu dx^2 / D_0, nu_s = refNu D_s / D_0, tau_s = nu_s / cs2 + 1/2."""
    ref_nu = 0.25 * (tau - 0.5)
    dt = ref_nu * dx * dx / d_pore[0]
    om_p = [1.0 / ((ref_nu if s == 0 else ref_nu * d_pore[s] / d_pore[0]) / 0.25 + 0.5) for s in range(len(d_pore))]
    om_b = [1.0 / (ref_nu * d_bio[s] / d_pore[0] / 0.25 + 0.5) for s in range(len(d_pore))]
    return ref_nu, dt, om_p, om_b


def test_carbonate_duct_parameters_and_unit_chain(clb, tmp_path):
    xml = case_files.run_dir(tmp_path, "carbonate_duct", case_files.carbonate_duct_map())
    c = clb.Case(xml)
    assert (c.get("nx"), c.get("ny"), c.get("nz")) == (22, 12, 10)
    assert c.get("dx") == pytest.approx(5e-6, rel=1e-15)
    assert c.get("Peclet") == 0 and c.get("tau") == 0.9
    assert c.get("n_substrates") == 4 and c.get("equilibrium") == 1
    # defaults of the reference where the file is silent
    assert c.get("ns_max_iT1") == 100000 and c.get("ns_converge_iT1") == 1e-8 and c.get("ns_converge_iT2") == 1e-6
    assert [c.get(f"substrate.{s}.left_type") for s in range(4)] == [0, 0, 2, 2]
    assert [c.get(f"substrate.{s}.right_type") for s in range(4)] == [1, 1, 2, 2]
    d_pore = [1e-9, 2e-9, 8e-10, 1.2e-9]
    d_bio = [5e-10, 1e-9, 4e-10, 6e-10]
    ref_nu, dt, om_p, om_b = unit_chain(0.9, 5e-6, d_pore, d_bio)
    assert c.get("refNu") == pytest.approx(ref_nu, rel=1e-15)
    assert c.get("ade_dt") == pytest.approx(dt, rel=1e-15)
    for s in range(4):
        assert c.get(f"substrate.{s}.omega_pore") == pytest.approx(om_p[s], rel=1e-15)
        assert c.get(f"substrate.{s}.omega_biofilm") == pytest.approx(om_b[s], rel=1e-15)


def test_biofilm_flow_parameters(clb, tmp_path):
    xml = case_files.run_dir(tmp_path, "biofilm_flow", case_files.biofilm_flow_map(clb))
    c = clb.Case(xml)
    assert c.get("nx") == 24 and c.get("Peclet") == 2 and c.get("delta_P") == 2e-5
    assert c.get("char_length") == pytest.approx(4.0)   # 8 um over dx = 2 um
    assert c.get("n_microbes") == 1 and c.get("microbe.0.code") == 3
    assert c.get("microbe.0.perm_ratio") == pytest.approx(0.25)
    with pytest.raises(clb.ClbError):
        c.get("ade_dt")  # needs the flow's pore velocity: known after setup


def rewrite(tmp_path, name, old, new):
    xml = case_files.run_dir(tmp_path, name, case_files.carbonate_duct_map())
    s = open(xml).read()
    assert old in s
    open(xml, "w").write(s.replace(old, new, 1))
    return xml


@pytest.mark.parametrize("old,new,msg", [
    ("<nx>20</nx>", "", "nx, ny and nz"),
    ("<left_boundary_type>Dirichlet</left_boundary_type>", "<left_boundary_type>Robin</left_boundary_type>",
     "Dirichlet, Neumann or closed"),
    ("<unit>um</unit>", "<unit>km</unit>", "m, mm or um"),
    ("<in_pore>1e-9</in_pore>", "<in_pore>0</in_pore>", "substrate 0 needs a positive pore diffusivity"),
    ("<tau>0.9</tau>", "<tau>3.5</tau>", "outside (0.5, 2]"),
    ("<initial_concentration>5e-4</initial_concentration>", "<initial_concentration>5e-4x</initial_concentration>",
     "not a number"),
    ("</parameters>", "", "unterminated"),
])
def test_errors_are_reported(clb, tmp_path, old, new, msg):
    xml = rewrite(tmp_path, "carbonate_duct", old, new)
    with pytest.raises(clb.ClbError, match=msg.replace("(", r"\(").replace(")", r"\)").replace("[", r"\[")
                       .replace("]", r"\]")):
        clb.Case(xml)


@pytest.mark.parametrize("old,new,msg", [
    ("<reaction_type>graphnet</reaction_type>", "<reaction_type>glpk</reaction_type>", "linear program"),
    ("<reaction_type>graphnet</reaction_type>", "<reaction_type>surrogate</reaction_type>", "no weights_file"),
    ("<reaction_type>graphnet</reaction_type>", "<reaction_type>graphnet_and_kinetics</reaction_type>",
     "a run-time law and a compiled one"),
    ("<reaction_type>graphnet</reaction_type>", "<reaction_type>quantum</reaction_type>", "is not defined"),
    ("<network_file>input/organism.gnn</network_file>", "", "names no network_file"),
    ("<enabled>true</enabled>", "<enabled>false</enabled>", "names no network_file"),
])
def test_rate_law_errors_are_reported(clb, tmp_path, old, new, msg):
    xml = case_files.run_dir(tmp_path, "graphnet_duct", case_files.graphnet_duct_map())
    text = open(xml).read()
    assert old in text
    open(xml, "w").write(text.replace(old, new))
    with pytest.raises(clb.ClbError, match=msg):
        clb.Case(xml)


def test_rate_law_blocks_parse(clb, tmp_path):
    xml = case_files.run_dir(tmp_path, "graphnet_duct", case_files.graphnet_duct_map())
    c = clb.Case(xml)
    assert c.get("graphnet") == 1 and c.get("symbolic") == 0 and c.get("microbe.0.reaction_type") == 9


def test_surrogate_case_parses(clb, tmp_path):
    c = clb.Case(case_files.surrogate_case(tmp_path, case_files.graphnet_duct_map()))
    assert c.get("surrogate") == 1 and c.get("microbe.0.reaction_type") == 3


def test_reference_examples_parse(clb):
    """Every CompLaB.xml the reference ships whose run lies on this path parses with its own
    values (checked when the reference checkout is named by CLB_REFERENCE_SRC)."""
    ref = os.environ.get("CLB_REFERENCE_SRC", "")
    files = sorted(glob.glob(os.path.join(ref, "examples", "*", "CompLaB.xml"))) if ref else []
    if not files:
        pytest.skip("no reference checkout named by CLB_REFERENCE_SRC")
    parsed = 0
    for f in files:
        try:
            c = clb.Case(f)
        except clb.ClbError as e:
            # microbes solved by finite differences or LBM are not on this path, nor are files
            # that leave out what a run off this path does not need
            assert "cellular-automaton" in str(e) or "FD" in str(e) or "missing" in str(e) or "needs" in str(e) \
                or "linear program" in str(e), (f, e)
            continue
        assert c.get("nx") >= 3 and c.get("n_substrates") >= 0
        parsed += 1
    assert parsed >= len(files) // 2
