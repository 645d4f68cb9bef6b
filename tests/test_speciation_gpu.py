"""FP64 Newton-Raphson speciation on the GPU against the oracle and the reference's own solver,
the speciation step inside the transport step, and the BF16 surrogate (training, gradients
against a CPU restatement, accuracy against Newton-Raphson, its use inside the transport step
and its gain over the solver on the 5 x 12 tableau)."""
import json
import os
import time

import numpy as np
import pytest

import workloads
from helpers import mixed_geometry

pytestmark = pytest.mark.gpu
GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "speciation.json")))


def handle(clb, S, logK, comp, n_species=None, tol=1e-10, prec=None):
    ns = S.shape[0]
    mat = np.full(4 * 4 * 4, 2, np.int8)
    D = clb.Domain(mat, 4, 4, 4, 0.8, ade_precision=clb.F64 if prec is None else prec)
    D.ade_init([dict(omega_pore=1.0, c0=1e-6)] * ns)
    D.speciation_setup(S, logK, comp, tol=tol)
    return D


@pytest.mark.parametrize("case", GOLD, ids=[c["name"] for c in GOLD])
def test_gpu_nr_matches_oracle_and_reference(clb, oracle, case):
    S = np.array(case["stoich"])
    cin = np.array(case["inputs"])
    D = handle(clb, S, case["logK"], case["component_species"])
    out, its = D.speciation_solve(cin)
    ora, conv, oits = oracle.eq_nr(S, case["logK"], case["component_species"], cin)
    pos = (cin @ S > 0).all(axis=1)
    np.testing.assert_allclose(out[pos], ora[pos], rtol=1e-9, atol=1e-20)
    ref = np.array(case["reference_outputs"])
    np.testing.assert_allclose(out[pos], ref[pos], rtol=2e-5, atol=1e-14)
    assert np.all(np.abs(its[pos] - oits[pos]) <= 1)


def test_speciation_step_in_transport_matches_oracle(clb, oracle):
    S, logK, comp = workloads.carbonate_tableau()
    shape = (14, 8, 7)
    mat = mixed_geometry(*shape, seed=21, biofilm=False)
    sp = [dict(omega_pore=1 / 0.9, left_type=0, right_type=1, left_bc=b, c0=c)
          for b, c in zip([2e-3, 1e-6, 1e-5, 5e-4], [1e-4, 3e-7, 2e-6, 1e-5])]
    rng = np.random.default_rng(3)
    u = np.zeros((3, mat.size))
    u[0] = 0.02 * rng.random(mat.size) * (mat == 2)
    D = clb.Domain(mat, *shape, 0.8, ade_precision=clb.F64)
    D.ade_init(sp)
    D.set_velocity(u)
    D.speciation_setup(S, logK, comp, tol=1e-10)
    D.set_speciation_mode(clb.SPEC_NR)
    O = oracle.OracleAde(mat, *shape, sp, u)
    O.set_speciation(S, logK, comp, tol=1e-10)
    D.ade_step(9)
    O.step(9)
    for s in range(4):
        # both sides stop Newton-Raphson at an absolute residual of 1e-10 on the totals
        np.testing.assert_allclose(D.concentration(s), O.concentration(s), rtol=1e-7, atol=1e-15)
    st = D.speciation_stats()
    assert st["solves"] > 0 and st["converged"] == st["solves"]


def bf16(a):
    a = np.asarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u >> 16) & 1) + 0x7FFF
    return (((u + r) >> 16) << 16).astype(np.uint32).view(np.float32).astype(np.float64)


def cpu_loss_grad(p, X, Y, ns):
    """The network's loss and parameter gradient in FP64, with every GEMM operand of the forward and
    the backward pass rounded to BF16 as the tensor cores see them (FP32 accumulation on the GPU)
    and the bias gradients from unrounded values."""
    W1 = p[:1024].reshape(64, 16); b1 = p[1024:1088]
    W2 = p[1088:5184].reshape(64, 64); b2 = p[5184:5248]
    W3 = p[5248:6272].reshape(16, 64); b3 = p[6272:6288]
    h1 = np.tanh(bf16(X) @ bf16(W1).T + b1)
    h2 = np.tanh(bf16(h1) @ bf16(W2).T + b2)
    y = bf16(h2) @ bf16(W3).T + b3
    n = X.shape[0]
    diff = np.zeros_like(y)
    diff[:, :ns] = y[:, :ns] - Y[:, :ns]
    loss = np.sum(diff ** 2)
    dy = 2 * diff / (n * ns)
    d2 = (bf16(dy) @ bf16(W3)) * (1 - h2 ** 2)
    d1 = (bf16(d2) @ bf16(W2)) * (1 - h1 ** 2)
    g = np.concatenate([(bf16(d1).T @ bf16(X)).ravel(), d1.sum(0), (bf16(d2).T @ bf16(h1)).ravel(), d2.sum(0),
                        (bf16(dy).T @ bf16(h2)).ravel(), dy.sum(0)])
    return loss, g


def test_surrogate_gradient_matches_cpu(clb):
    S, logK, comp = workloads.tableau_5x12()
    D = handle(clb, S, logK, comp)
    rng = np.random.default_rng(5)
    n_par = clb.lib().clb_surrogate_param_count()
    p = (0.2 * rng.standard_normal(n_par)).astype(np.float32)
    p[1024:1088] = 0.05 * rng.standard_normal(64)
    p[np.arange(1024).reshape(64, 16)[:, 5:].ravel()] = 0.0   # inputs beyond the 5 components are padding
    sc = np.concatenate([-np.ones(16), np.ones(16), -np.ones(16), np.ones(16)]).astype(np.float32)
    D.surrogate_params(p, sc)
    X = np.zeros((300, 16), np.float32)
    X[:, :5] = rng.uniform(-1, 1, size=(300, 5))
    Y = np.zeros((300, 16), np.float32)
    Y[:, :12] = rng.uniform(-1, 1, size=(300, 12))
    g, loss = D.surrogate_gradient(X, Y)
    loss_c, g_c = cpu_loss_grad(p.astype(np.float64), X.astype(np.float64), Y.astype(np.float64), 12)
    assert loss == pytest.approx(loss_c, rel=1e-4)
    scale = np.abs(g_c).max()
    assert np.max(np.abs(g - g_c)) < 2e-3 * scale
    assert np.dot(g, g_c) / (np.linalg.norm(g) * np.linalg.norm(g_c)) > 0.99999


def test_surrogate_training_is_deterministic(clb):
    """Gradients are summed per block and then across blocks in a fixed order (no atomics), and the
    validation loss likewise, so two trainings from the same seed give the same parameters bit for
    bit."""
    S, logK, comp = workloads.carbonate_tableau()
    out = []
    for _ in range(2):
        D = handle(clb, S, logK, comp)
        D.surrogate_train([-5, -9, -8, -6], [-2, -5, -4, -3], n_samples=20000, epochs=3, batch=1024, patience=8,
                          learning_rate=3e-3, seed=5)
        out.append(D.surrogate_params()[0])
        D.close()
    np.testing.assert_array_equal(out[0], out[1])


@pytest.fixture(scope="module")
def trained(clb):
    S, logK, comp = workloads.carbonate_tableau()
    D = handle(clb, S, logK, comp)
    lo, hi = [-5, -9, -8, -6], [-2, -5, -4, -3]
    rep = D.surrogate_train(lo, hi, n_samples=200000, epochs=60, batch=1024, patience=8, learning_rate=3e-3, seed=11)
    return D, S, logK, comp, lo, hi, rep


def test_surrogate_trains_and_matches_newton(trained, oracle):
    D, S, logK, comp, lo, hi, rep = trained
    print("training:", rep)
    assert rep["val_mse"] < 1e-3
    states = workloads.species_states(4000, 4, np.array(lo), np.array(hi), seed=99)
    states = states[(states @ S > 0).all(axis=1)]
    nr, _ = D.speciation_solve(states)
    D.surrogate_set_check(0.02, 0)  # the network alone
    raw, _ = D.surrogate_predict(states, residual_check=False)
    D.surrogate_set_check(0.02, 2)  # with the two-step Newton polish
    pol, acc = D.surrogate_predict(states, residual_check=True)
    r_raw = np.abs(raw / nr - 1)
    r_pol = np.abs(pol / nr - 1)
    print("network alone: median rel err %.2e, p95 %.2e; polished: median %.2e, max %.2e, accepted %.3f"
          % (np.median(r_raw), np.percentile(r_raw, 95), np.median(r_pol), r_pol.max(), acc.mean()))
    assert np.median(r_raw) < 0.1
    assert np.percentile(r_pol[acc], 99) <= 1e-3
    assert acc.mean() > 0.8


def transport_times(clb, S, logK, comp, params, scaling, sp, shape, seed):
    """Device time of 20 transport steps with Newton-Raphson speciation and with the surrogate and
    its Newton polish, and the fraction of solves the surrogate kept."""
    mat = mixed_geometry(*shape, seed=seed, biofilm=False)
    times, used = {}, {}
    for mode in (clb.SPEC_NR, clb.SPEC_MLP_NR):
        D = clb.Domain(mat, *shape, 0.8, ade_precision=clb.F32)
        D.ade_init(sp)
        D.speciation_setup(S, logK, comp, tol=1e-10)
        D.surrogate_params(params, scaling)
        D.surrogate_set_check(0.02, 2)
        D.set_speciation_mode(mode)
        D.ade_step(4)
        D.sync()
        s0 = D.speciation_stats()
        ts = []
        for _ in range(3):
            t0 = time.perf_counter()
            D.ade_step(20)
            D.sync()
            ts.append(time.perf_counter() - t0)
        s1 = D.speciation_stats()
        times[mode] = min(ts)
        used[mode] = (s1["surrogate_used"] - s0["surrogate_used"]) / max(1, s1["solves"] - s0["solves"])
        D.close()
    return times, used


def test_surrogate_kept_in_transport(clb, trained):
    """The two-component carbonate system inside the transport step: the surrogate answers nearly
    every solve. (Newton-Raphson on two components converges in a few cheap iterations in the
    fixed-shape build, so the surrogate is not expected to be faster here; its gain is shown on
    the 5 x 12 tableau below.)"""
    D0, S, logK, comp, lo, hi, rep = trained
    params, scaling = D0.surrogate_params()
    sp = [dict(omega_pore=1 / 0.9, left_type=0, right_type=1, left_bc=b, c0=c)
          for b, c in zip([2e-3, 1e-6, 1e-5, 5e-4], [1e-4, 3e-7, 2e-6, 1e-5])]
    times, used = transport_times(clb, S, logK, comp, params, scaling, sp, (34, 32, 32), 25)
    print("20 transport steps: Newton-Raphson %.2f ms, surrogate + polish %.2f ms (surrogate kept on %.3f)"
          % (times[clb.SPEC_NR] * 1e3, times[clb.SPEC_MLP_NR] * 1e3, used[clb.SPEC_MLP_NR]))
    assert used[clb.SPEC_MLP_NR] > 0.5


def test_surrogate_gain_over_newton(clb):
    """What the trained network gains over the method without it, inside the transport step (no
    host transfer involved): the 5-component, 12-species tableau on a rough fracture (the
    benchmark's precipitation configuration at half size, its species fed and initially present as
    there), the surrogate trained on the GPU from Newton-Raphson solves of the run's own voxel
    states jittered by up to 0.6 decades; with it (and its two-step Newton polish and residual
    check) a step takes less time than with Newton-Raphson alone, and it answers most solves."""
    cfg = workloads.fracture192_carbonate(
        lambda nx, ny, nz: clb.geom_generate("fracture", nx, ny, nz, aperture=12.0, roughness=0.3, seed=1004,
                                             walls="none"), scale=0.5)
    S, logK, comp = cfg["S"], cfg["logK"], cfg["comp"]
    ns = S.shape[0]

    def domain():
        D = clb.Domain(cfg["mat"], *cfg["shape"], cfg["tau"], ade_precision=clb.F32)
        D.ade_init(cfg["species"])
        D.speciation_setup(S, logK, comp, tol=1e-10)
        D.set_speciation_mode(clb.SPEC_NR)
        D.ade_step(10)
        return D

    T = domain()
    T.surrogate_train([-6.0] * ns, [-2.5] * ns, n_samples=200000, epochs=60, batch=1024, patience=8,
                      learning_rate=3e-3, seed=1004, from_domain=True, jitter=0.6)
    params, scaling = T.surrogate_params()
    T.close()
    times, used = {}, {}
    for mode in (clb.SPEC_NR, clb.SPEC_MLP_NR):
        D = domain()
        D.surrogate_params(params, scaling)
        D.surrogate_set_check(0.02, 2, 1e-6)
        D.set_speciation_mode(mode)
        D.ade_step(2)
        D.sync()
        s0 = D.speciation_stats()
        ts = []
        for _ in range(3):
            t0 = time.perf_counter()
            D.ade_step(10)
            D.sync()
            ts.append(time.perf_counter() - t0)
        s1 = D.speciation_stats()
        times[mode] = min(ts)
        used[mode] = (s1["surrogate_used"] - s0["surrogate_used"]) / max(1, s1["solves"] - s0["solves"])
        D.close()
    print("10 transport steps (5 x 12): Newton-Raphson %.2f ms, surrogate + polish %.2f ms (surrogate kept on %.3f)"
          % (times[clb.SPEC_NR] * 1e3, times[clb.SPEC_MLP_NR] * 1e3, used[clb.SPEC_MLP_NR]))
    assert used[clb.SPEC_MLP_NR] > 0.5
    assert times[clb.SPEC_MLP_NR] < times[clb.SPEC_NR]


def test_surrogate_with_fallback_in_transport(clb, oracle, trained):
    D0, S, logK, comp, lo, hi, rep = trained
    params, scaling = D0.surrogate_params()
    shape = (14, 8, 7)
    mat = mixed_geometry(*shape, seed=21, biofilm=False)
    sp = [dict(omega_pore=1 / 0.9, left_type=0, right_type=1, left_bc=b, c0=c)
          for b, c in zip([2e-3, 1e-6, 1e-5, 5e-4], [1e-4, 3e-7, 2e-6, 1e-5])]
    results = {}
    for mode in (clb.SPEC_NR, clb.SPEC_MLP_NR):
        D = clb.Domain(mat, *shape, 0.8, ade_precision=clb.F64)
        D.ade_init(sp)
        D.speciation_setup(S, logK, comp, tol=1e-10)
        D.surrogate_params(params, scaling)
        D.surrogate_set_check(0.02, 2)
        D.set_speciation_mode(mode)
        D.ade_step(12)
        results[mode] = (np.array([D.concentration(s) for s in range(4)]), D.speciation_stats())
    a, st = results[clb.SPEC_MLP_NR]
    b, _ = results[clb.SPEC_NR]
    print("surrogate step stats:", st)
    assert st["surrogate_used"] + st["fallbacks"] == st["solves"]
    open_ = (mat == 2)
    # a kept surrogate answer meets a 1e-6 relative mass balance; species agree to 1e-4
    np.testing.assert_allclose(a[:, open_], b[:, open_], rtol=1e-4)
    assert st["surrogate_used"] > 0.5 * st["solves"]


def test_surrogate_trained_on_the_runs_own_states(clb):
    """Training data drawn from the domain's own voxel states (the solves the method generates):
    the surrogate then answers nearly every voxel of that run, to Newton-Raphson accuracy."""
    S, logK, comp = workloads.carbonate_tableau()
    shape = (16, 9, 8)
    mat = mixed_geometry(*shape, seed=23, biofilm=False)
    sp = [dict(omega_pore=1 / 0.9, left_type=0, right_type=1, left_bc=b, c0=c)
          for b, c in zip([2e-3, 1e-6, 1e-5, 5e-4], [1e-4, 3e-7, 2e-6, 1e-5])]
    out = {}
    for mode in (clb.SPEC_NR, clb.SPEC_MLP_NR):
        D = clb.Domain(mat, *shape, 0.8, ade_precision=clb.F64)
        D.ade_init(sp)
        D.speciation_setup(S, logK, comp, tol=1e-10)
        D.set_speciation_mode(clb.SPEC_NR)
        D.ade_step(6)
        if mode == clb.SPEC_MLP_NR:
            rep = D.surrogate_train([-8] * 4, [-2] * 4, n_samples=100000, epochs=40, batch=1024, patience=8,
                                    learning_rate=3e-3, seed=3, from_domain=True, jitter=0.5)
            assert rep["n_train"] > 50000
            D.surrogate_set_check(0.02, 2, 1e-6)
        D.set_speciation_mode(mode)
        s0 = D.speciation_stats()
        D.ade_step(6)
        s1 = D.speciation_stats()
        out[mode] = (np.array([D.concentration(s) for s in range(4)]),
                     (s1["surrogate_used"] - s0["surrogate_used"]) / max(1, s1["solves"] - s0["solves"]))
    a, used = out[clb.SPEC_MLP_NR]
    b, _ = out[clb.SPEC_NR]
    print("surrogate used on", used)
    assert used > 0.9
    open_ = mat == 2
    np.testing.assert_allclose(a[:, open_], b[:, open_], rtol=1e-4)
