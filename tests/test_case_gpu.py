"""CompLaB.xml cases run end to end through the library (clb_case_setup + clb_case_run) against the
FP64 oracle set up from the same description: the geometry file, the unit chain, the boundary types,
the equilibrium tableau, the flow with its Peclet rescale."""
import numpy as np
import pytest

import case_files
from helpers import rel_l2

pytestmark = pytest.mark.gpu


def species_from(c):
    n = int(c.get("n_substrates"))
    return [dict(omega_pore=c.get(f"substrate.{s}.omega_pore"), omega_biofilm=c.get(f"substrate.{s}.omega_biofilm"),
                 mobile=int(c.get(f"substrate.{s}.mobile")), left_type=int(c.get(f"substrate.{s}.left_type")),
                 right_type=int(c.get(f"substrate.{s}.right_type")), left_bc=c.get(f"substrate.{s}.left_bc"),
                 right_bc=c.get(f"substrate.{s}.right_bc"), c0=c.get(f"substrate.{s}.c0")) for s in range(n)]


def ghosted(inner):
    nx, ny, nz = inner.shape
    full = np.empty((nx + 2, ny, nz), np.int8)
    full[1:-1] = inner
    full[0], full[-1] = inner[0], inner[-1]
    return full.ravel()


def test_carbonate_duct_runs_like_the_oracle(clb, oracle, tmp_path):
    inner = case_files.carbonate_duct_map()
    xml = case_files.run_dir(tmp_path, "carbonate_duct", inner)
    c = clb.Case(xml)
    D = c.setup(clb.F64, clb.F64)
    out = tmp_path / "vti"
    out.mkdir()
    rep = c.run(D, output_dir=str(out))
    assert rep["iterations"] == 300
    # one file per substrate every save_VTK_interval (100) iterations
    assert len(list(out.glob("*.vti"))) == 4 * 3 and (out / "HCO3_0000300.vti").exists()
    mat = ghosted(inner)
    np.testing.assert_array_equal(D.material(), mat)
    sp = species_from(c)
    O = oracle.OracleAde(mat, int(c.get("nx")), int(c.get("ny")), int(c.get("nz")), sp, np.zeros(3 * mat.size))
    S = np.array([[1, 0], [0, 1], [1, -1], [1, 1]], float)
    O.set_speciation(S, [0.0, 0.0, -10.33, 6.35], [0, 1], tol=1e-10)
    O.step(300)
    for s in range(4):
        # both sides stop Newton-Raphson at an absolute residual of 1e-10 on the totals, so the
        # minor species (CO3 at log K -10.33) agree to a few 1e-7 after 300 steps (3.2e-7 measured)
        cg, co = D.concentration(s), O.concentration(s)
        assert rel_l2(cg, co) < 2e-6, s
    assert D.concentration(2).max() > 0  # the complexes formed


def test_biofilm_flow_case_sets_up_like_the_reference(clb, oracle, tmp_path):
    """Flow at a target Peclet number: the pressure drop is rescaled, PoreMeanU is taken over the
    pore and biofilm voxels (complab.cpp:1128-1150), refNu = PoreMeanU L / Pe, ade_dt and every
    relaxation rate follow (complab.cpp:1221-1253); the flow field equals the oracle's at the drop
    used; the coupled run through the case schedule completes."""
    inner = case_files.biofilm_flow_map(clb)
    xml = case_files.run_dir(tmp_path, "biofilm_flow", inner)
    c = clb.Case(xml)
    D = c.setup(clb.F64, clb.F64)
    mat = ghosted(inner)
    nx, ny, nz = int(c.get("nx")), int(c.get("ny")), int(c.get("nz"))
    dp = c.get("delta_P_used")
    assert dp != 2e-5  # rescaled
    OF = oracle.OracleFlow(mat, nx, ny, nz, 0.8, dp, bio_codes=(3, 4), perm_ratio=(0.25, 0.25))
    OF.solve(40000, 1e-7)
    u = OF.velocity()
    assert rel_l2(D.velocity(), u) < 1e-9
    # PoreMeanU (the re-solved field: the whole interior), refNu, ade_dt, omegas
    P = ny * nz
    norm = np.sqrt((u ** 2).sum(0))
    pmu = norm[P:-P].mean()
    assert c.get("pore_mean_u") == pytest.approx(pmu, rel=1e-8)
    ref_nu = pmu * c.get("char_length") / 2.0
    assert c.get("refNu") == pytest.approx(ref_nu, rel=1e-8)
    dx = 2e-6
    assert c.get("ade_dt") == pytest.approx(ref_nu * dx * dx / 1e-9, rel=1e-8)
    assert c.get("substrate.1.omega_pore") == pytest.approx(1 / (ref_nu * 2.0 / 0.25 + 0.5), rel=1e-8)
    assert c.get("substrate.1.omega_biofilm") == pytest.approx(1 / (ref_nu * 0.8 / 0.25 + 0.5), rel=1e-8)
    # a rate law of the run's own (dual Monod in physical units per second, dt = ade_dt)
    D.set_kinetics(clb.LAW_DUAL_MONOD, [2e-3, 0.05, 0.4, 1e-6], c.get("ade_dt"))
    b0 = D.biomass(0).sum()
    rep = c.run(D)
    assert rep["iterations"] == 60 and rep["flow_resolves"] >= 0
    assert np.isfinite(D.concentration(0)).all() and D.biomass(0).sum() > b0


def test_graphnet_case_binds_its_networks(clb, tmp_path):
    """reaction_type graphnet and the <graphnet> block: the case binds the organism's network and
    the abiotic one at set-up (files beside the XML), and its run equals a run of the same case
    with the block switched off and the two networks bound by hand, bit for bit."""
    import os
    xml = case_files.run_dir(tmp_path, "graphnet_duct", case_files.graphnet_duct_map())
    c = clb.Case(xml)
    assert c.get("graphnet") == 1 and c.get("microbe.0.reaction_type") == 9
    D = c.setup(clb.F64, clb.F64)
    out, _ = D.graph_network_eval(0, np.full((1, 4), 0.3))
    assert out.shape == (1, 5)
    rep = c.run(D)
    assert rep["iterations"] == 80
    # the same description with the block off, networks bound through the library's entry points
    text = open(xml).read().replace("<enabled>true</enabled>", "<enabled>false</enabled>").replace(
        "<reaction_type>graphnet</reaction_type>", "<reaction_type>kinetics</reaction_type>")
    xml2 = os.path.join(os.path.dirname(xml), "manual.xml")
    open(xml2, "w").write(text)
    c2 = clb.Case(xml2)
    assert c2.get("graphnet") == 0
    D2 = c2.setup(clb.F64, clb.F64)
    inp = os.path.join(os.path.dirname(xml), "input")
    D2.set_graph_network(os.path.join(inp, "organism.gnn"), ["A", "B", "C", "D"], 0)
    D2.set_graph_network(os.path.join(inp, "abiotic.gnn"), ["A", "B", "C", "D"], -1)
    c2.run(D2)
    for s in range(4):
        np.testing.assert_array_equal(D.concentration(s), D2.concentration(s))
    np.testing.assert_array_equal(D.biomass(0), D2.biomass(0))
    b0 = case_files.graphnet_duct_map()
    assert np.abs(D.biomass(0)).sum() != 60.0 * (b0 == 3).sum()  # the network grew or decayed it


def test_surrogate_case_binds_its_network(clb, tmp_path):
    """reaction_type surrogate and the <surrogate> block: the case binds the organism's .srg network
    with the microbe block's uptake parameters (half-saturation constants, fba_maximum_uptake_flux,
    biomass_molar_mass, decay_coefficient), and its run equals the same case with the organism bound
    by hand, bit for bit."""
    import os
    xml = case_files.surrogate_case(tmp_path, case_files.graphnet_duct_map())
    c = clb.Case(xml)
    D = c.setup(clb.F64, clb.F64)
    out, _ = D.surrogate_eval(0, np.full((1, 2), 5.0))
    assert out.shape == (1, 3)
    b0 = D.biomass(0).copy()
    c.run(D)
    text = open(xml).read().replace("<reaction_type>surrogate</reaction_type>", "<reaction_type>kinetics</reaction_type>")
    text = text.replace("<surrogate>\n        <enabled>true</enabled>", "<surrogate>\n        <enabled>false</enabled>")
    xml2 = os.path.join(os.path.dirname(xml), "manual_srg.xml")
    open(xml2, "w").write(text)
    c2 = clb.Case(xml2)
    assert c2.get("surrogate") == 0
    D2 = c2.setup(clb.F64, clb.F64)
    inp = os.path.join(os.path.dirname(xml), "input")
    D2.set_surrogate_organism(os.path.join(inp, "organism.srg"), ["A", "B", "C", "D"], 0, [0.05, 0.1, 0.02, 0.2],
                              [10, 5, 0, 0], 24.6, 2e-6)
    D2.set_graph_network(os.path.join(inp, "abiotic.gnn"), ["A", "B", "C", "D"], -1)
    c2.run(D2)
    for s in range(4):
        np.testing.assert_array_equal(D.concentration(s), D2.concentration(s))
    np.testing.assert_array_equal(D.biomass(0), D2.biomass(0))
    assert np.abs(D.biomass(0) - b0).max() > 1e-9
