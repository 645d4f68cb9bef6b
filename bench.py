#!/usr/bin/env python
"""Throughput of the D3Q19 flow step on the 256x128x128 overlapping-sphere pack (porosity 0.35,
grain radius U[3, 8], tau 0.7), FP32 populations, one GPU per rank.

A step is one collide-and-stream of the whole lattice (one launch of the AA kernel). MLUPS
counts open (collide) voxels; the all-voxel figure is reported alongside. Only the collide/stream nodes
are stored (sparse layout), so the FP32 lattice is about the size of L2: the benchmark flushes L2
between timed steps and times each step with its own event pair.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Side measurements in the same JSON line (rank 0, one GPU; --no-extra skips them):
  "d3q7"       fused transport of the 256^3 pack, 8 species, 2 microbes, FP32: species-voxel
               updates per second and its HBM roofline;
  "precision"  FP64 / FP32 / FP16-shifted flow throughput and the velocity, permeability and
               concentration errors of the reduced-precision paths against the FP64 path;
  "speciation" the 5 x 12 tableau in transport: Newton-Raphson against the trained surrogate
               (time per step, solves per second, speed-up, error against Newton-Raphson);
  "ensemble"   96 uneven domains with flow and 3 species advanced by the batched, graph-replayed
               steps: domain-steps per second and aggregate MLUPS.

Multi-GPU: the domain does not shard on this path (single-domain solver); each rank advances
its own replica and the value is the sum over ranks divided by the slowest rank's time.
The reference arm times the FP64 CPU restatement of the reference path (the reference itself
needs Palabos, which is not available) on all host cores, on a bounded x-slab of the same map.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "complab3d-gems_b200"))

import numpy as np  # noqa: E402

METRIC = "MLUPS (D3Q19+D3Q7) & % HBM roofline; mixed vs FP64 GPU at stated L2 err; CPU ref"
PEAK_FALLBACK = 6650.0


def args_():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=4000)
    p.add_argument("--warmup", type=int, default=50)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--precision", default="f32", choices=["f64", "f32", "f16s"])
    p.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    p.add_argument("--no-extra", action="store_true", help="skip the D3Q7, precision and speciation legs")
    p.add_argument("--scale", type=float, default=1.0, help="shrink the workload (testing only)")
    p.add_argument("--no-autotune", action="store_true",
                   help="keep the library's default kernel variants (profiling runs: timings under a profiler "
                        "would mislead the autotuner)")
    p.add_argument("--leg", choices=["d3q7", "precision", "speciation", "ensemble"],
                   help="run only this side measurement (with --scale for d3q7) and print its JSON; "
                        "a small case for profilers, not a bench line")
    return p.parse_args()


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return PEAK_FALLBACK, "fallback"


def max_over_ranks(torch, ms, world, device):
    """The slowest rank's time: every rank takes part in the same all-reduce (MAX)."""
    if world == 1:
        return ms
    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(n_open, steps, ms_max, world):
    """Whole-job MLUPS of `world` replicas of the same domain: every rank updates n_open nodes per
    step; the job takes the slowest rank's time."""
    return world * n_open * steps / (ms_max * 1e-3) / 1e6


def step_kernels(tuned, precision):
    """Names of the two AA-step kernels the flow step ran (the autotuner's choice, else the
    library's defaults: tiled even step, pipelined odd step for 4- and 8-byte storage)."""
    choice = tuned.split("->")[-1] if "->" in tuned else ("tma=1,pipe" if precision != "f16s" else "tma=1,minb=3")
    even = "k_flow_even_tma" if "tma=1" in choice else "k_flow_aa<even>"
    odd = "k_flow_odd_pipe" if "pipe" in choice else "k_flow_aa<odd>"
    return f"{even} + {odd} (AA even/odd steps, mean per launch)"


def traffic_per_launch(kernel_key):
    """DRAM bytes per launch from the committed ncu summary (profiles/traffic.txt)."""
    path = os.path.join(ROOT, "profiles", "traffic.txt")
    try:
        for line in open(path):
            parts = line.split()
            if len(parts) >= 2 and parts[0] == kernel_key:
                return float(parts[1])
    except OSError:
        pass
    return None


class ClockSampler:
    """Polls SM clock and clock-event reasons through NVML while the timed region runs."""

    REASONS = {0x1: "gpu_idle", 0x2: "applications_clocks_setting", 0x4: "sw_power_cap", 0x8: "hw_slowdown",
               0x10: "sync_boost", 0x20: "sw_thermal_slowdown", 0x40: "hw_thermal_slowdown",
               0x80: "hw_power_brake_slowdown", 0x100: "display_clock_setting"}

    def __init__(self, index):
        self.samples, self.reasons, self.ok = [], 0, False
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nv = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByIndex(index)
            self.max = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
            self.ok = True
        except Exception:
            self.max = None
        self._stop = threading.Event()

    def _run(self):
        while not self._stop.is_set():
            try:
                self.samples.append(self.nv.nvmlDeviceGetClockInfo(self.h, self.nv.NVML_CLOCK_SM))
                self.reasons |= self.nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
            except Exception:
                pass
            time.sleep(0.002)

    def __enter__(self):
        if self.ok:
            self.t = threading.Thread(target=self._run, daemon=True)
            self.t.start()
        return self

    def __exit__(self, *a):
        if self.ok:
            self._stop.set()
            self.t.join()

    def summary(self):
        if not self.ok or not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max, "reasons": ["unavailable"]}
        names = [v for k, v in self.REASONS.items() if self.reasons & k and v != "gpu_idle"]
        return {"sm_mhz": statistics.median(self.samples), "sm_max_mhz": self.max, "reasons": names,
                "samples": len(self.samples)}


def cpu_name():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def slab(mat, shape, nx_s):
    nx, ny, nz = shape
    m = mat.reshape(nx, ny, nz)[:nx_s].copy()
    m[-1] = m[-2]
    return m.ravel(), (nx_s, ny, nz)


def oracle_mlups(mat, shape, tau, dp, min_seconds, min_steps, max_steps):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    threads = oracle.max_threads()
    oracle.set_threads(threads)
    O = oracle.OracleFlow(mat, *shape, tau, dp)
    n_open = int(np.sum(mat == 2))
    O.step(1)
    steps, t0 = 0, time.perf_counter()
    while steps < max_steps and (steps < min_steps or time.perf_counter() - t0 < min_seconds):
        O.step(1)
        steps += 1
    dt = time.perf_counter() - t0
    return n_open * steps / dt / 1e6, threads, steps, dt


def run_reference(a, cfg):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    mat, shape = slab(cfg["mat"], cfg["shape"], 18)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    threads = oracle.max_threads()
    oracle.set_threads(threads)
    O = oracle.OracleFlow(mat, *shape, cfg["tau"], cfg["delta_p"])
    n_open = int(np.sum(mat == 2))
    O.step(max(1, a.warmup))
    t0 = time.perf_counter()
    O.step(a.steps)
    dt = time.perf_counter() - t0
    v = n_open * a.steps / dt / 1e6
    sample = f"x-slab 16+2 planes of the 256x128x128 map ({shape[0]}x{shape[1]}x{shape[2]}), FP64, {a.steps} steps"
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": "MLUPS", "n_gpus": a.gpus, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": dt / a.steps * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded sphere pack)",
        "config": {"workload": cfg["name"] + " (x-slab sample)", "nx": shape[0], "ny": shape[1], "nz": shape[2],
                   "open_voxels": n_open},
        "cpu_baseline": {"value": v, "unit": "MLUPS", "cores": threads, "kind": "port", "cpu": cpu_name(),
                         "sample": sample},
        "e2e": {"value": v, "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def timed_steps(torch, stream, step, steps, warmup):
    """Device time of `steps` calls of step() on `stream` (one event pair around all of them)."""
    step(warmup)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    step(steps)
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1)


def bench_d3q7(clb, workloads, torch, local, peak, steps=60, warmup=5, scale=1.0):
    """Fused transport of the 256^3 sphere pack with 8 species and 2 biofilm microbes (dual Monod),
    FP32 populations; the lattice (1.5 GB) is far larger than L2, so no flush is needed."""
    cfg = workloads.pack256cube_8species(scale=scale)
    nx, ny, nz = cfg["shape"]
    mat = cfg["mat"]
    D = clb.Domain(mat, nx, ny, nz, cfg["tau"], flow_precision=clb.F32, ade_precision=clb.F32,
                   bio_codes=cfg["bio_codes"], perm_ratio=cfg["perm_ratio"], device=local)
    stream = torch.cuda.Stream()
    D.set_stream(stream.cuda_stream)
    D.flow_init(cfg["delta_p"])
    D.flow_step(400)
    D.ade_init(cfg["species"])
    D.couple_velocity()
    D.set_biomass(cfg["biomass"])
    D.set_kinetics(cfg["law"], cfg["params"], cfg["dt"])
    ms = timed_steps(torch, stream, D.ade_step, steps, warmup)
    # the same step with the thermodynamic gate on the biotic rates (species 0 + 1 -> 2)
    D.set_thermo_gate(species=(0, 1, 2), nu=(-1.0, -1.0, 1.0), dG0=-20.0, atp=0.25, dGatp=50.0)
    ms_gate = timed_steps(torch, stream, D.ade_step, steps, warmup)
    D.set_thermo_gate()
    S = len(cfg["species"])
    n_open = int(np.count_nonzero((mat != 0) & (mat != 1)))
    per = ms / steps
    M = cfg["biomass"].shape[0]
    alg_node = S * 2 * 7 * 4 + 3 * 4 + 1 + M * 8
    achieved = alg_node * n_open / (per * 1e-3) / 1e9
    D.close()
    return {"workload": cfg["name"] + ", FP32 populations, dual-Monod kinetics fused",
            "mlups_d3q7": S * n_open * steps / (ms * 1e-3) / 1e6, "unit": "species x open-voxel updates / s (1e6)",
            "ms_per_step": per, "thermo_gate_ms_per_step": ms_gate / steps, "open_voxels": n_open, "species": S,
            "steps": steps,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "algorithmic_bytes_per_node": alg_node, "kernel": "k_ade_aa (all species fused)"}}


def bench_precision(clb, workloads, torch, local, steps=300, warmup=20):
    """FP64 / FP32 / FP16-shifted storage: flow throughput and velocity / permeability error on the
    256x128x128 pack (3000 steps from the same state), and the transport error on the 64x32x32
    pack (flow to 1e-6, 2000 steps of decaying solute), each against the FP64 GPU path, which
    matches the FP64 oracle to 1e-12."""
    out = {}
    cfg = workloads.pack256x128x128()
    nx, ny, nz = cfg["shape"]
    ref_u = ref_k = None
    for name, prec in (("f64", clb.F64), ("f32", clb.F32), ("f16s", clb.F16S)):
        D = clb.Domain(cfg["mat"], nx, ny, nz, cfg["tau"], flow_precision=prec, device=local)
        stream = torch.cuda.Stream()
        D.set_stream(stream.cuda_stream)
        D.flow_init(cfg["delta_p"])
        D.autotune(10)
        ms = timed_steps(torch, stream, D.flow_step, steps, warmup)
        D.flow_step(3000 - steps - warmup)
        st = D.flow_stats(cfg["char_length"])
        u = D.velocity()
        n_open = st["bgk_nodes"]
        r = {"flow_mlups": n_open * steps / (ms * 1e-3) / 1e6, "permeability": st["permeability"]}
        if ref_u is None:
            ref_u, ref_k = u, st["permeability"]
        else:
            r["velocity_rel_l2_vs_f64"] = float(np.linalg.norm(u - ref_u) / np.linalg.norm(ref_u))
            r["velocity_rel_max_vs_f64"] = float(np.abs(u - ref_u).max() / np.abs(ref_u).max())
            r["permeability_rel_err_vs_f64"] = abs(st["permeability"] / ref_k - 1)
        out[name] = r
        D.close()
    out["f32"]["speedup_vs_f64"] = out["f32"]["flow_mlups"] / out["f64"]["flow_mlups"]
    out["f16s"]["speedup_vs_f64"] = out["f16s"]["flow_mlups"] / out["f64"]["flow_mlups"]
    c1 = workloads.pack64x32x32_decay()
    nx, ny, nz = c1["shape"]
    ref_c = None
    for name, prec in (("f64", clb.F64), ("f32", clb.F32), ("f16s", clb.F16S)):
        D = clb.Domain(c1["mat"], nx, ny, nz, c1["tau"], flow_precision=prec, ade_precision=prec, device=local)
        D.flow_init(c1["delta_p"])
        it = D.flow_solve(200000, c1["eps"], allow_unconverged=True)
        D.ade_init(c1["species"])
        D.couple_velocity()
        D.set_kinetics(c1["law"], c1["params"], c1["dt"])
        D.ade_step(c1["ade_steps"])
        c = D.concentration(0)
        u = D.velocity()
        if ref_c is None:
            ref_c, ref_u1 = c, u
            out[name]["pack64_flow_iterations"] = it
        else:
            out[name]["pack64_concentration_rel_l2_vs_f64"] = float(np.linalg.norm(c - ref_c) / np.linalg.norm(ref_c))
            out[name]["pack64_velocity_rel_l2_vs_f64"] = float(np.linalg.norm(u - ref_u1) / np.linalg.norm(ref_u1))
        D.close()
    return out


def bench_speciation(clb, workloads, torch, local, steps=10):
    """Equilibrium speciation of the 5-component, 12-species tableau inside the transport step on a
    96^3 pack: Newton-Raphson (FP64) against the BF16 surrogate with a two-step Newton polish and
    Newton-Raphson fallback. The surrogate is trained on the GPU from Newton-Raphson solves of the
    states the run itself generates (1e6 samples of the domain's voxels after 20 steps, each
    species scaled by 10^U(-0.6, 0.6)). Speciation time = step time with it minus step time
    without; error = max relative species difference after one step from the same state (open
    voxels), against Newton-Raphson. The component H+ (species 0) is kept dominant so every
    component total is positive (the reference clamps non-positive totals to 1e-30)."""
    S, logK, comp = workloads.tableau_5x12()
    ns = S.shape[0]
    mat, shape = workloads.sphere_pack_domain(96, 96, 96, 0.40, 3.0, 6.0, seed=1004)
    rng = np.random.default_rng(1004)
    sp = [dict(omega_pore=1 / 0.9, left_type=clb.DIRICHLET, right_type=clb.NEUMANN,
               left_bc=float(10 ** rng.uniform(-6, -4)), c0=float(10 ** rng.uniform(-6, -4))) for _ in range(ns)]
    sp[0]["c0"], sp[0]["left_bc"] = 3e-3, 2e-3
    D = clb.Domain(mat, *shape, 0.8, ade_precision=clb.F32, device=local)
    stream = torch.cuda.Stream()
    D.set_stream(stream.cuda_stream)
    D.ade_init(sp)
    D.speciation_setup(S, logK, comp, tol=1e-10)
    D.set_speciation_mode(clb.SPEC_NR)
    D.ade_step(20)
    t_train = time.perf_counter()
    rep = D.surrogate_train([-6.0] * ns, [-2.5] * ns, n_samples=1000000, epochs=60, batch=1024, patience=8,
                            learning_rate=3e-3, seed=1004, from_domain=True, jitter=0.6)
    t_train = time.perf_counter() - t_train
    D.surrogate_set_check(0.02, 2, 1e-6)
    n_open = int(np.count_nonzero(mat == 2))
    times = {}
    used = 0.0
    for mode in (clb.SPEC_OFF, clb.SPEC_NR, clb.SPEC_MLP_NR):
        D.set_speciation_mode(mode)
        s0 = D.speciation_stats()
        times[mode] = timed_steps(torch, stream, D.ade_step, steps, 2) / steps
        s1 = D.speciation_stats()
        if mode == clb.SPEC_MLP_NR:
            used = (s1["surrogate_used"] - s0["surrogate_used"]) / max(1, s1["solves"] - s0["solves"])
    # accuracy: one step from the same state under each mode
    conc0 = [D.ade_populations(s) for s in range(ns)]
    res = {}
    for mode in (clb.SPEC_NR, clb.SPEC_MLP_NR):
        for s in range(ns):
            D.set_ade_populations(s, conc0[s])
        D.set_speciation_mode(mode)
        D.ade_step(1)
        res[mode] = np.array([D.concentration(s) for s in range(ns)])
    open_ = (mat == 2)
    a, b = res[clb.SPEC_MLP_NR][:, open_], res[clb.SPEC_NR][:, open_]
    rel = np.abs(a / np.where(b == 0, 1, b) - 1)
    D.close()
    t_nr = times[clb.SPEC_NR] - times[clb.SPEC_OFF]
    t_ml = times[clb.SPEC_MLP_NR] - times[clb.SPEC_OFF]
    return {"workload": "96^3 sphere pack, 5 components x 12 species tableau, FP32 transport, FP64 speciation",
            "open_voxels": n_open, "nr_ms_per_step": t_nr, "surrogate_ms_per_step": t_ml,
            "nr_solves_per_s": n_open / (t_nr * 1e-3), "surrogate_solves_per_s": n_open / (t_ml * 1e-3),
            "speedup": t_nr / t_ml, "max_rel_err_vs_nr": float(rel.max()), "p99_rel_err_vs_nr": float(np.percentile(rel, 99)),
            "surrogate_used_fraction": used,
            "training": {"seconds": t_train, "val_mse": rep["val_mse"], "epochs": rep["epochs"],
                         "n_train": rep["n_train"], "source": "the run's own voxel states, jitter 0.6 decades"}}


def bench_ensemble(clb, workloads, torch, local, steps=200):
    """96 independent uneven domains (the parameter-sweep configuration), FP32, each with a D3Q19
    flow and 3 D3Q7 species with Monod kinetics, advanced by the batched steps (one launch per
    lattice and step for all domains, pairs of steps replayed from a CUDA graph) after the
    batch autotuner, against the same domains stepped one after another."""
    cfg = workloads.ensemble_uneven_packs()
    doms = []
    for d in cfg["domains"]:
        nx, ny, nz = d["shape"]
        D = clb.Domain(d["mat"], nx, ny, nz, d["tau"], flow_precision=clb.F32, ade_precision=clb.F32, device=local)
        D.flow_init(d["delta_p"])
        D.flow_step(20)
        D.ade_init(d["species"])
        D.couple_velocity()
        D.set_kinetics(d["law"], d["params"], d["dt"])
        doms.append(D)
    B = clb.Batch(doms)
    tuned = B.autotune(10)
    nf, nt = B.counts()
    B.step(4)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    B.step(steps)
    dt = time.perf_counter() - t0
    # the same domains one by one (each call enqueues its own launches)
    k = 20
    t1 = time.perf_counter()
    for D in doms:
        D.flow_step(k)
        D.ade_step(k)
    for D in doms:
        D.sync()
    dt1 = (time.perf_counter() - t1) / k
    B.close()
    for D in doms:
        D.close()
    n = len(doms)
    upd = nf + 3 * nt
    return {"workload": cfg["name"] + ", FP32", "domains": n, "flow_nodes": nf, "transport_nodes": nt,
            "steps": steps, "ms_per_step": dt / steps * 1e3, "domain_steps_per_s": n * steps / dt,
            "aggregate_mlups": upd * steps / dt / 1e6,
            "unit": "domain-steps / s; MLUPS = flow node + species x transport node updates / s (1e6)",
            "one_by_one_ms_per_step": dt1 * 1e3, "speedup_vs_one_by_one": dt1 / (dt / steps),
            "autotune": tuned, "timing": "host clock around the batched steps (one synchronisation)"}


def main():
    a = args_()
    import clb
    import workloads

    if a.impl == "reference":
        run_reference(a, workloads.pack256x128x128(scale=a.scale))
        return

    import torch

    if a.leg:
        local = int(os.environ.get("LOCAL_RANK", "0"))
        torch.cuda.set_device(local)
        fn = {"d3q7": lambda: bench_d3q7(clb, workloads, torch, local, peaks()[0], steps=10, warmup=3, scale=a.scale),
              "precision": lambda: bench_precision(clb, workloads, torch, local),
              "speciation": lambda: bench_speciation(clb, workloads, torch, local),
              "ensemble": lambda: bench_ensemble(clb, workloads, torch, local)}[a.leg]
        print(json.dumps({"leg": a.leg, "scale": a.scale, a.leg: fn()}))
        return
    cfg = workloads.pack256x128x128(scale=a.scale)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    prec = {"f64": clb.F64, "f32": clb.F32, "f16s": clb.F16S}[a.precision]
    es = {"f64": 8, "f32": 4, "f16s": 2}[a.precision]
    nx, ny, nz = cfg["shape"]
    mat = cfg["mat"]

    D = clb.Domain(mat, nx, ny, nz, cfg["tau"], flow_precision=prec, device=local)
    stream = torch.cuda.Stream()
    D.set_stream(stream.cuda_stream)
    D.flow_init(cfg["delta_p"])
    tuned = "defaults" if a.no_autotune else D.autotune(20)
    st = D.flow_stats()
    n_open, n_active = st["bgk_nodes"], st["active_nodes"]

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    D.flow_step(a.warmup)
    D.sync()
    barrier()
    torch.cuda.synchronize()
    # The compacted FP32 lattice (~120 MB) is about the size of L2, so L2 is flushed between
    # timed steps on the same stream: a 256 MB buffer is written and then read back, so the L2
    # ends up holding clean lines of that buffer (none of the lattice, and no dirty lines whose
    # write-back the next step would pay for). Only the steps are timed (one event pair each).
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    flush_sum = torch.empty((), dtype=torch.int64, device="cuda")
    ev0 = [torch.cuda.Event(enable_timing=True) for _ in range(a.steps)]
    ev1 = [torch.cuda.Event(enable_timing=True) for _ in range(a.steps)]
    with ClockSampler(local) as clocks:
        for s in range(a.steps):
            ev0[s].record(stream)
            D.flow_step(1)
            ev1[s].record(stream)
            with torch.cuda.stream(stream):
                flush.fill_(s & 255)
                torch.sum(flush.view(torch.int64), dim=0, out=flush_sum)
        ev1[-1].synchronize()
    torch.cuda.synchronize()
    barrier()
    ms = sum(e0.elapsed_time(e1) for e0, e1 in zip(ev0, ev1))
    del flush, flush_sum
    ms = max_over_ranks(torch, ms, world, "cuda")
    per_step = ms / a.steps
    value = replica_throughput(n_open, a.steps, ms, world)
    all_vox = world * nx * ny * nz * a.steps / (ms * 1e-3) / 1e6

    # roofline of the step kernel: algorithmic bytes = 2 * 19 * sizeof(storage) per open node
    alg = 2 * 19 * es * n_open
    peak, peak_kind = peaks()
    achieved = alg / (per_step * 1e-3) / 1e9
    key = f"k_flow_aa_{a.precision}_pack256x128x128"
    tr = traffic_per_launch(key)
    roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": tr, "peak_source": peak_kind, "algorithmic_bytes_per_launch": alg,
            "kernel": step_kernels(tuned, a.precision)}

    D.close()
    del D
    torch.cuda.synchronize()
    # end to end through the C ABI with host buffers: create (the material map goes in from pinned
    # host memory) + init (the layout is built on the device) + the same steps + the velocity back
    # into pinned host memory, in the storage's precision
    k_e2e = a.steps
    udt = torch.float64 if a.precision == "f64" else torch.float32
    mat_host = torch.empty(mat.size, dtype=torch.int8, pin_memory=True).numpy()
    mat_host[:] = mat
    u_host = torch.empty(3 * mat.size, dtype=udt, pin_memory=True).numpy()
    # the whole job three times; the median job time is reported
    t_jobs, phases = [], []
    for _ in range(3):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        E = clb.Domain(mat_host, nx, ny, nz, cfg["tau"], flow_precision=prec, device=local)
        t1 = time.perf_counter()
        E.flow_init(cfg["delta_p"])
        E.sync()
        t2 = time.perf_counter()
        E.flow_step(k_e2e)
        E.sync()
        t3 = time.perf_counter()
        u = E.velocity(u_host.dtype, out=u_host)
        t4 = time.perf_counter()
        t_jobs.append(t4 - t0)
        phases.append({"create": 1e3 * (t1 - t0), "init": 1e3 * (t2 - t1), "steps": 1e3 * (t3 - t2),
                       "velocity_to_host": 1e3 * (t4 - t3)})
        E.close()
        del E
    t_e2e = statistics.median(t_jobs)
    job_phases = phases[t_jobs.index(t_e2e)]
    e2e_val = world * n_open * k_e2e / t_e2e / 1e6
    h2d = mat_host.nbytes  # the compacted layout is built on the device from the map
    d2h = u.nbytes

    extra = {}
    if rank == 0 and world == 1 and not a.no_extra and a.scale == 1.0:
        for key, fn in (("d3q7", lambda: bench_d3q7(clb, workloads, torch, local, peak)),
                        ("precision", lambda: bench_precision(clb, workloads, torch, local)),
                        ("speciation", lambda: bench_speciation(clb, workloads, torch, local)),
                        ("ensemble", lambda: bench_ensemble(clb, workloads, torch, local))):
            try:
                extra[key] = fn()
            except Exception as exc:  # a failed side measurement must not hide the headline line
                extra[key] = {"error": f"{type(exc).__name__}: {exc}"}
            torch.cuda.synchronize()

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu:
        v, threads, steps, dt = oracle_mlups(mat, cfg["shape"], cfg["tau"], cfg["delta_p"], 12.0, 2, 400)
        cpu = {"value": v, "unit": "MLUPS", "cores": threads, "kind": "port", "cpu": cpu_name(),
               "sample": f"{steps} FP64 steps of the full 258x128x128 map in {dt:.1f} s (OpenMP)"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "MLUPS", "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": a.precision, "data": "synthetic (seeded sphere pack)",
            "config": {"workload": cfg["name"] + f", D3Q19 IncBGK, {a.precision.upper()} populations",
                       "nx": nx, "ny": ny, "nz": nz, "open_voxels": n_open, "active_nodes": n_active,
                       "all_voxel_mlups": all_vox, "l2": "flushed between timed steps (256 MB write, then read back); "
                       "compacted lattice %.0f MB" % (19 * es * n_active / 1e6), "parallelism": f"replicas x{world}",
                       "autotune": tuned},
            "roofline": roof,
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_val, "unit": "MLUPS", "h2d_bytes_per_step": h2d / k_e2e,
                    "d2h_bytes_per_step": d2h / k_e2e,
                    "note": "one job through the C ABI: create + init + K steps + velocity to host, wall clock; "
                            "median of 3 jobs", "job_seconds": t_jobs,
                    "median_job_phases_ms": job_phases},
            "gpu_launches": a.steps,
            "clocks": clocks.summary(),
        }
        line.update(extra)
        print(json.dumps(line))
    if world > 1:
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
