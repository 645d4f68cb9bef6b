"""The BASELINE configurations against the FP64 oracle at their own sizes.

Config 1 (the reference's CPU-runnable case) at full size: the 64x32x32 sphere pack (+2 ghost
planes), tau 0.8, pressure drop 1e-4, flow to the ValueTracer criterion 1e-6, then 2000 steps of
the decaying solute (k = 1e-3, clamped) with a Dirichlet inlet and a Neumann outlet, FP64 on the
GPU and in the oracle: iteration count within 1, velocity and concentration within 1e-10 relative
(L2 and max).

Config 4 at reduced size: the reference's fracture generator (aperture 12, roughness 0.3), the
5-component 12-species tableau solved per voxel by FP64 Newton-Raphson inside every transport
step, an immobile mineral that grows with the saturation Omega of two aqueous species, voxels that
seal at the full mineral density (checked every 10 steps; the deposit starts uniform in
[0, full) so voxels seal one after another) with the flow re-solved through the new bounce-back
voxels; the sealed set bit-exact and the fields close to the oracle's."""
import numpy as np
import pytest

import workloads
from helpers import rel_l2

pytestmark = pytest.mark.gpu


def test_config1_full_size_f64_matches_oracle(clb, oracle):
    w = workloads.pack64x32x32_decay()
    nx, ny, nz = w["shape"]
    assert (nx, ny, nz) == (66, 32, 32)
    D = clb.Domain(w["mat"], nx, ny, nz, w["tau"], flow_precision=clb.F64, ade_precision=clb.F64)
    D.flow_init(w["delta_p"])
    it_g, conv = D.flow_solve(200000, w["eps"])
    O = oracle.OracleFlow(w["mat"], nx, ny, nz, w["tau"], w["delta_p"])
    it_o = O.solve(200000, w["eps"])
    assert conv and abs(it_g - it_o) <= 1, (it_g, it_o)
    ug, uo = D.velocity(), O.velocity()
    assert rel_l2(ug, uo) < 1e-10
    assert np.max(np.abs(ug - uo)) < 1e-10 * np.max(np.abs(uo))
    D.ade_init(w["species"])
    D.couple_velocity()
    D.set_kinetics(w["law"], w["params"], w["dt"])
    D.ade_step(w["ade_steps"])
    A = oracle.OracleAde(w["mat"], nx, ny, nz, w["species"], uo)
    A.set_kinetics(w["law"], w["params"], w["dt"])
    A.step(w["ade_steps"])
    cg, co = D.concentration(0), A.concentration(0)
    assert rel_l2(cg, co) < 1e-10
    assert np.max(np.abs(cg - co)) < 1e-10 * np.max(np.abs(co))
    print(f"config 1: flow iterations {it_g} / {it_o}, velocity rel L2 {rel_l2(ug, uo):.2e}, "
          f"concentration rel L2 {rel_l2(cg, co):.2e}")


def config4_reduced():
    S, logK, comp = workloads.tableau_5x12()
    ns = S.shape[0]
    nxi, ny, nz = 30, 24, 24
    mat = clb_mod().geom_generate("fracture", nxi, ny, nz, aperture=12.0, roughness=0.3, seed=1004, walls="none")
    # the generator's codes: 0 solid rock, 2 pore; rock is the reference's solid (NoDynamics on the
    # flow lattice, bounce-back for the species); add the ghost planes
    mat, shape = workloads.add_ghost_planes(mat, nxi, ny, nz), (nxi + 2, ny, nz)
    rng = np.random.default_rng(1004)
    sp = [dict(omega_pore=1 / 0.9, left_type=0, right_type=1, left_bc=float(10 ** rng.uniform(-5, -3.5)),
               c0=float(10 ** rng.uniform(-6, -4))) for _ in range(ns)]
    sp[0]["c0"], sp[0]["left_bc"] = 3e-3, 2e-3
    for s in (1, 2):   # the two mineral-forming components, supersaturated in the domain and the feed
        sp[s]["c0"], sp[s]["left_bc"] = 2e-3, 2e-3
    sp.append(dict(omega_pore=1.0, mobile=0, left_type=1, right_type=1, c0=0.0))   # the mineral (immobile)
    nu = [0.0] * (ns + 1)
    nu[1], nu[2] = 1.0, 1.0
    mineral = [2e-6, -6.0, ns] + nu        # k, log10 Ksp, mineral species, nu
    # mineral already deposited, uniform in [0, full) over the pore voxels: voxels seal one after
    # another as it grows, scattered through the fracture rather than a whole plane at once
    full = 1e-3
    m0 = np.random.default_rng(5).uniform(0.0, full, mat.size) * (mat == 2)
    return S, logK, comp, mat, shape, sp, mineral, full, m0


def clb_mod():
    import clb
    return clb


def test_config4_reduced_speciation_precipitation_and_resolve(clb, oracle):
    S, logK, comp, mat, shape, sp, mineral, full, m0 = config4_reduced()
    nx, ny, nz = shape
    ns = S.shape[0]
    D = clb.Domain(mat, nx, ny, nz, 0.8, flow_precision=clb.F64, ade_precision=clb.F64)
    D.flow_init(1e-4)
    D.flow_step(300)
    OF = oracle.OracleFlow(mat, nx, ny, nz, 0.8, 1e-4)
    OF.step(300)
    D.ade_init(sp)
    D.couple_velocity()
    O = oracle.OracleAde(mat, nx, ny, nz, sp, OF.velocity())
    D.speciation_setup(S, logK, comp, tol=1e-10)
    D.set_speciation_mode(clb.SPEC_NR)
    O.set_speciation(S, logK, comp, tol=1e-10)
    D.set_abiotic_kinetics(clb.LAW_MINERAL, mineral, 0)
    O.set_abiotic(5, mineral, 0)
    D.set_concentration(ns, m0)
    O.set_immobile(ns, m0)
    D.precip_setup(ns, full, seal_flow=1, flow_max_iterations=80, flow_eps=0.0)
    O.set_precip(ns, full, precip_code=0)
    OF.set_dynamics(127, 0, 0.0)  # sealed voxels: bounce-back on the flow lattice
    total_sealed = 0
    for rnd in range(8):
        D.ade_step(10)
        O.step(10)
        a = D.geometry_update(allow_unconverged=True)
        b = O.geometry_update()
        assert a == b, (rnd, a, b)
        total_sealed += a[0]
        np.testing.assert_array_equal(D.material(), O.material())
        if a[0] or a[1]:
            fm = mat.copy()
            fm[(O.material() == 0) & (mat != 0)] = 127
            OF.set_material(fm)
            OF.step(80)
            O.set_velocity(OF.velocity())
        np.testing.assert_allclose(D.velocity(), OF.velocity(), rtol=0, atol=1e-12)
    for s in range(ns + 1):
        cg, co = D.concentration(s), O.concentration(s)
        assert rel_l2(cg, co) < 1e-7, s
    st = D.speciation_stats()
    assert st["solves"] > 0 and st["converged"] == st["solves"]
    assert total_sealed > 0  # the run does seal voxels
    print(f"config 4 (reduced): {total_sealed} voxels sealed in 80 steps")
