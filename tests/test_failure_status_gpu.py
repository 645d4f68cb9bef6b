"""The run-stopping statuses of the reference, raised by host-side injection only (no device fault):
non-finite concentrations in a transport step, a diverged flow solve and non-finite biomass return
CLB_NONFINITE (complab.cpp:2796, 3116-3117); a flow path sealed shut returns CLB_PERCOLATION_LOST
at the re-solve's iteration cap (complab.cpp:3106-3113). After each, the handle still answers."""
import numpy as np
import pytest

from helpers import mixed_geometry

pytestmark = pytest.mark.gpu

NONFINITE, PERCOLATION_LOST = 3, 4
SP = [dict(omega_pore=1 / 0.9, omega_biofilm=1 / 0.7, left_type=0, right_type=1, left_bc=1.0, c0=0.0),
      dict(omega_pore=1.0, left_type=1, right_type=1, c0=0.3)]


@pytest.mark.parametrize("prec", ["F64", "F32", "F16S"])
def test_nan_population_stops_the_transport(clb, prec):
    shape = (14, 8, 9)
    mat = mixed_geometry(*shape, seed=8)
    D = clb.Domain(mat, *shape, 0.8, ade_precision=getattr(clb, prec), bio_codes=(3, 4), perm_ratio=(0.3, 0.3))
    D.ade_init(SP)
    D.ade_step(3)
    D.sync()  # clean so far
    g = D.ade_populations(1)
    pore = np.flatnonzero(mat == 2)
    g[2, pore[len(pore) // 2]] = np.nan
    D.set_ade_populations(1, g)
    D.ade_step(1)
    with pytest.raises(clb.ClbError) as e:
        D.sync()
    assert e.value.status == NONFINITE
    with pytest.raises(clb.ClbError) as e:
        D.ade_step(1)
    assert e.value.status == NONFINITE
    # the handle still answers, and the reductions count the bad voxels
    assert D.reduce()["nonfinite"] >= 1
    # a clean state clears it
    g[2, pore[len(pore) // 2]] = 0.0
    D.set_ade_populations(1, np.nan_to_num(D.ade_populations(1)))
    D.set_ade_populations(0, np.nan_to_num(D.ade_populations(0)))
    D.ade_step(2)
    D.sync()


def test_infinite_population_stops_the_transport(clb):
    shape = (12, 8, 8)
    mat = mixed_geometry(*shape, seed=9)
    D = clb.Domain(mat, *shape, 0.8, ade_precision=clb.F32, bio_codes=(3, 4), perm_ratio=(0.3, 0.3))
    D.ade_init(SP)
    g = D.ade_populations(0)
    g[0, np.flatnonzero(mat == 2)[7]] = np.inf
    D.set_ade_populations(0, g)
    D.ade_step(1)
    with pytest.raises(clb.ClbError) as e:
        D.sync()
    assert e.value.status == NONFINITE


def test_diverged_flow_solve_is_nonfinite(clb):
    shape = (16, 8, 8)
    mat = mixed_geometry(*shape, seed=10, biofilm=False)
    D = clb.Domain(mat, *shape, 0.8, flow_precision=clb.F64)
    D.flow_init(1e-4)
    D.flow_step(10)
    f = D.flow_populations()
    f[5, np.flatnonzero(mat == 2)[11]] = np.nan
    D.set_flow_populations(f)
    with pytest.raises(clb.ClbError) as e:
        D.flow_solve(700, 1e-6)
    assert e.value.status == NONFINITE
    D.flow_init(1e-4)  # a fresh start works
    D.flow_step(3)
    assert np.isfinite(D.velocity()).all()


def sealed_duct(nx=40, ny=8, nz=8, seal_at=20):
    m = np.full((nx, ny, nz), 2, np.int8)
    m[:, 0, :] = m[:, -1, :] = 1
    m[:, :, 0] = m[:, :, -1] = 1
    m[seal_at] = 1  # a wall across the whole section: no path from inlet to outlet
    return m.ravel()


@pytest.mark.parametrize("prec,cap", [("F64", 800), ("F32", 8000)])
def test_sealed_path_loses_percolation(clb, prec, cap):
    """The reference flags a lost percolation path only when the re-solve stops at its cap with
    the outlet plane's mean u_x at or below 1e-12 (complab.cpp:3092-3113); a sealed duct whose
    energy settles (FP64 reaches a constant round-off energy after about 1000 iterations) counts as
    converged there and the run goes on. So the FP64 case stops at 800 iterations, while the
    energy still falls by orders of magnitude per window and the outlet's mean u_x is near 4e-15
    (the oracle's values); FP32 never settles below its round-off noise."""
    shape = (40, 8, 8)
    D = clb.Domain(sealed_duct(), *shape, 0.8, flow_precision=getattr(clb, prec))
    D.flow_init(1e-4)
    with pytest.raises(clb.ClbError) as e:
        D.flow_solve(cap, 1e-9)
    assert e.value.status == PERCOLATION_LOST
    # the same duct open: the solve converges and the outlet flows
    open_duct = sealed_duct()
    open_duct.reshape(shape)[20] = 2
    open_duct.reshape(shape)[20, 0, :] = open_duct.reshape(shape)[20, -1, :] = 1
    open_duct.reshape(shape)[20, :, 0] = open_duct.reshape(shape)[20, :, -1] = 1
    E = clb.Domain(open_duct, *shape, 0.8, flow_precision=getattr(clb, prec))
    E.flow_init(1e-4)
    it, conv = E.flow_solve(40000, 1e-7)
    assert conv
    assert E.flow_stats()["darcy_outlet_ux"] > 1e-9


def test_nonfinite_biomass_stops_the_automaton(clb):
    shape = (16, 10, 9)
    mat = mixed_geometry(*shape, seed=11)
    D = clb.Domain(mat, *shape, 0.8, ade_precision=clb.F64, bio_codes=(3, 4), perm_ratio=(0.3, 0.3))
    D.ade_init(SP)
    bio = np.zeros((2, mat.size))
    bio[0, mat == 3] = 20.0
    bio[1, mat == 4] = 30.0
    D.set_biomass(bio)
    D.ca_setup(100.0, 0.1, 5)
    st, sweeps, changed = D.ca_step()
    assert st == 0
    bad = bio.copy()
    bad[0, np.flatnonzero(mat == 3)[0]] = np.nan
    D.set_biomass(bad)
    with pytest.raises(clb.ClbError) as e:
        D.ca_step()
    assert e.value.status == NONFINITE
