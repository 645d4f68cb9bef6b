"""The coupled driver (clb_run) against the same iterations made through the step-by-step calls,
and its flow re-solves' convergence tracer kept across re-solves as the reference keeps its
in-loop ValueTracer (complab.cpp:2166, ns_convg2, never reset)."""
import numpy as np
import pytest

from helpers import mixed_geometry

pytestmark = pytest.mark.gpu

SPECIES = [
    dict(omega_pore=1 / 0.9, omega_biofilm=1 / 0.7, left_type=0, right_type=1, left_bc=1.0, c0=0.3),
    dict(omega_pore=1 / 0.62, omega_biofilm=1 / 0.56, left_type=0, right_type=1, left_bc=0.8, c0=0.2),
]


def biofilm_domain(clb, shape, seed, prec):
    mat = mixed_geometry(*shape, seed=seed)
    rng = np.random.default_rng(seed)
    bio = np.zeros((2, mat.size))
    bio[0, mat == 3] = rng.uniform(80, 99.9, size=(mat == 3).sum())
    bio[1, mat == 4] = rng.uniform(80, 99.9, size=(mat == 4).sum())
    D = clb.Domain(mat, *shape, 0.8, flow_precision=prec, ade_precision=prec, bio_codes=(3, 4), perm_ratio=(0.3, 0.3))
    D.flow_init(2e-4)
    D.flow_step(200)
    D.ade_init(SPECIES)
    D.couple_velocity()
    D.set_biomass(bio)
    D.set_kinetics(3, [2e-3, 0.1, 0.4, 1e-6], 1.0)  # fast growth: the automaton pushes within the run
    D.ca_setup(100.0, 0.1, 7)
    return D


@pytest.mark.parametrize("prec", ["F64", "F32"])
def test_run_equals_the_step_by_step_calls(clb, prec):
    """clb_run enqueues the automaton's steps without reading them back each iteration (and the
    species dynamics refresh acts only after a step that changed the mask); the fields after the
    run equal those of ade_step + ca_step + refresh_dynamics called iteration by iteration."""
    shape = (20, 12, 10)
    p = getattr(clb, prec)
    A = biofilm_domain(clb, shape, 31, p)
    B = biofilm_domain(clb, shape, 31, p)
    n = 150
    rep = A.run(n, ca=True, ade_update_interval=1)
    sweeps = changes = 0
    for _ in range(n):
        B.ade_step(1)
        st, sw, ch = B.ca_step()
        sweeps += sw
        if ch:
            changes += 1
            B.refresh_dynamics(species=True, flow=False)
    assert rep["iterations"] == n
    assert rep["ca_sweeps"] == sweeps and rep["mask_changes"] == changes
    assert sweeps > 0  # the automaton did push
    np.testing.assert_array_equal(A.material(), B.material())
    np.testing.assert_array_equal(A.ca_total(), B.ca_total())
    np.testing.assert_array_equal(A.ca_age(), B.ca_age())
    for m in range(2):
        np.testing.assert_array_equal(A.biomass(m), B.biomass(m))
    for s in range(2):
        np.testing.assert_array_equal(A.concentration(s), B.concentration(s))


def test_resolve_keeps_the_tracer_window(clb):
    """The first re-solve of a run fills an empty window (at least its 500 values); a later
    re-solve with nothing changed in between converges on its first step, because the window it
    starts from already satisfies the criterion."""
    shape = (24, 12, 10)
    mat = mixed_geometry(*shape, seed=33, biofilm=False)
    D = clb.Domain(mat, *shape, 0.8, flow_precision=clb.F64, ade_precision=clb.F64)
    D.flow_init(1e-4)
    D.flow_solve(20000, 1e-6)
    D.ade_init(SPECIES)
    D.couple_velocity()
    r1 = D.run(20, resolve_every=10, flow_max_iterations=20000, flow_eps=1e-6)
    assert r1["flow_resolves"] == 2
    r2 = D.run(20, resolve_every=10, flow_max_iterations=20000, flow_eps=1e-6)
    assert r2["flow_resolves"] == 2 and r2["flow_iterations"] == 2
    assert r1["flow_iterations"] >= 500 + 1
