"""Ensembles of uneven domains advanced by the batched steps (the persistent schedule: a table of
(step, domain, lattice, tile) items walked by one launch per few steps; or one launch per lattice
and step; launches replayed from CUDA graphs) against the same domains stepped one by one: the
populations must agree bit for bit, in FP64, FP32 and FP16-shifted storage."""
import numpy as np
import pytest

import workloads

pytestmark = pytest.mark.gpu


def build(clb, cfg, prec):
    out = []
    for d in cfg["domains"]:
        nx, ny, nz = d["shape"]
        D = clb.Domain(d["mat"], nx, ny, nz, d["tau"], flow_precision=prec, ade_precision=prec)
        D.flow_init(d["delta_p"])
        D.flow_step(30)
        D.ade_init(d["species"])
        D.couple_velocity()
        D.set_kinetics(d["law"], d["params"], d["dt"])
        out.append(D)
    return out


def assert_same(A, B):
    for a, b in zip(A, B):
        np.testing.assert_array_equal(a.flow_populations(), b.flow_populations())
        for s in range(a.S):
            np.testing.assert_array_equal(a.ade_populations(s), b.ade_populations(s))


@pytest.mark.parametrize("prec", ["F64", "F32"])
def test_batch_matches_single_domains(clb, prec):
    cfg = workloads.ensemble_uneven_packs(n_domains=7, seed=11, scale=0.5)
    p = getattr(clb, prec)
    A = build(clb, cfg, p)
    B = build(clb, cfg, p)
    batch = clb.Batch(B)
    for n, flow, tr in ((10, True, True), (7, True, False), (5, False, True), (1, True, True)):
        for D in A:
            if flow:
                D.flow_step(n)
            if tr:
                D.ade_step(n)
        batch.step(n, flow=flow, transport=tr)
    assert_same(A, B)
    fa, ta = batch.counts()
    assert fa == sum(D.flow_stats()["active_nodes"] for D in B)
    batch.close()


def test_batch_autotune_then_matches(clb):
    cfg = workloads.ensemble_uneven_packs(n_domains=5, seed=12, scale=0.5)
    A = build(clb, cfg, clb.F32)
    B = build(clb, cfg, clb.F32)
    batch = clb.Batch(B)
    rep = batch.autotune(4)
    assert "flow" in rep and "transport" in rep
    nf = B[0].flow_stats()["iterations"] - A[0].flow_stats()["iterations"]
    nt = B[0].reduce()["ade_iterations"] - A[0].reduce()["ade_iterations"]
    assert nf > 0 and nt > 0
    for D in A:
        D.flow_step(nf)
        D.ade_step(nt)
    batch.step(12)
    for D in A:
        D.flow_step(12)
        D.ade_step(12)
    assert_same(A, B)
    batch.close()


def test_batch_rejects_mixed_parity(clb):
    cfg = workloads.ensemble_uneven_packs(n_domains=2, seed=13, scale=0.5)
    B = build(clb, cfg, clb.F32)
    B[1].ade_step(1)
    batch = clb.Batch(B)
    with pytest.raises(clb.ClbError):
        batch.step(2)
    batch.close()


@pytest.mark.parametrize("prec,sched", [
    ("F32", dict(persistent=False)),
    ("F32", dict(persistent=False, staged_flow=True)),
    ("F64", dict(persistent=False, staged_flow=True)),
    ("F32", dict(tile=256, lag=1, steps_per_launch=2)),
    ("F32", dict(tile=1024, lag=3, steps_per_launch=8, ctas_per_sm=8)),
    ("F32", dict(tile=2048, lag=8, steps_per_launch=2, ctas_per_sm=6)),
    ("F64", dict(tile=512, lag=2, steps_per_launch=4)),
    ("F16S", dict(tile=4096, lag=100, steps_per_launch=6)),
])
def test_batch_schedules_match_single_domains(clb, prec, sched):
    """Every schedule of the batched steps (per-lattice launches; persistent item tables with tiles
    of 256 to 4096 nodes, lags from 1 domain (a domain's next step right behind its last) to more
    than the ensemble, 2 to 8 steps per launch, graph replays and remainder launches) gives the
    populations of stepping each domain on its own, bit for bit."""
    cfg = workloads.ensemble_uneven_packs(n_domains=9, seed=21, scale=0.5)
    p = getattr(clb, prec)
    A = build(clb, cfg, p)
    B = build(clb, cfg, p)
    batch = clb.Batch(B)
    batch.schedule(**sched)
    got = batch.get_schedule()
    assert got["persistent"] == sched.get("persistent", True)
    assert got["staged_flow"] == sched.get("staged_flow", False)
    for n, flow, tr in ((17, True, True), (9, True, False), (6, False, True), (3, True, True)):
        for D in A:
            if flow:
                D.flow_step(n)
            if tr:
                D.ade_step(n)
        batch.step(n, flow=flow, transport=tr)
    assert_same(A, B)
    batch.close()


def test_batch_schedule_rejects_bad_settings(clb):
    cfg = workloads.ensemble_uneven_packs(n_domains=2, seed=22, scale=0.5)
    B = build(clb, cfg, clb.F32)
    batch = clb.Batch(B)
    for bad in (dict(tile=300), dict(lag=0), dict(steps_per_launch=3), dict(steps_per_launch=10), dict(ctas_per_sm=5)):
        with pytest.raises(clb.ClbError):
            batch.schedule(**bad)
    batch.close()


def test_batch_staged_flow_needs_four_byte_storage(clb):
    cfg = workloads.ensemble_uneven_packs(n_domains=2, seed=23, scale=0.5)
    B = build(clb, cfg, clb.F16S)
    batch = clb.Batch(B)
    with pytest.raises(clb.ClbError):
        batch.schedule(persistent=False, staged_flow=True)
    assert batch.get_schedule()["staged_flow"] is False
    batch.close()


def test_persistent_wait_limit_reports_timeout(clb):
    """A dependency wait of the persistent schedule that reaches its limit gives up on the device:
    with a limit far below a step's duration, waits that find their dependency still in progress
    give up, the launch skips its remaining items, the step returns CLB_TIMEOUT and the device
    stays usable (the same batch steps again once the limit is back)."""
    cfg = workloads.ensemble_uneven_packs(n_domains=9, seed=24, scale=0.5)
    B = build(clb, cfg, clb.F32)
    batch = clb.Batch(B)
    batch.schedule(tile=256, lag=1, steps_per_launch=8)
    batch.set_wait_limit(1)
    with pytest.raises(clb.ClbError) as err:
        batch.step(8)
    assert clb.STATUS[err.value.status] == "TIMEOUT" and "wait" in str(err.value)
    batch.set_wait_limit(2_000_000_000)
    batch.step(8)
    batch.close()
    for D in B:
        D.close()
