#!/usr/bin/env python
"""Throughput of the D3Q19 flow step on the 256x128x128 overlapping-sphere pack (BASELINE
config 2: porosity 0.35, grain radius U[3, 8], tau 0.7), FP32 populations, one GPU per rank.

A step is one collide-and-stream of the whole lattice (one launch of the AA kernel). MLUPS
counts open (collide) voxels; the all-voxel figure is reported alongside. Only the collide/stream nodes
are stored (sparse layout), so the FP32 lattice is about the size of L2: the benchmark flushes L2
between timed steps and times each step with its own event pair.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

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
    p.add_argument("--scale", type=float, default=1.0, help="shrink the workload (testing only)")
    return p.parse_args()


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return PEAK_FALLBACK, "fallback"


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


def main():
    a = args_()
    import clb
    import workloads

    cfg = workloads.config2(scale=a.scale)
    if a.impl == "reference":
        run_reference(a, cfg)
        return

    import torch

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
    tuned = D.autotune(20)
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
    # timed steps by writing a 256 MB buffer on the same stream; only the steps are timed
    # (one event pair per step).
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    ev0 = [torch.cuda.Event(enable_timing=True) for _ in range(a.steps)]
    ev1 = [torch.cuda.Event(enable_timing=True) for _ in range(a.steps)]
    with ClockSampler(local) as clocks:
        for s in range(a.steps):
            ev0[s].record(stream)
            D.flow_step(1)
            ev1[s].record(stream)
            with torch.cuda.stream(stream):
                flush.fill_(s & 255)
        ev1[-1].synchronize()
    torch.cuda.synchronize()
    barrier()
    ms = sum(e0.elapsed_time(e1) for e0, e1 in zip(ev0, ev1))
    del flush
    if world > 1:
        t = torch.tensor([ms], device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms = float(t.item())
    per_step = ms / a.steps
    value = world * n_open * a.steps / (ms * 1e-3) / 1e6
    all_vox = world * nx * ny * nz * a.steps / (ms * 1e-3) / 1e6

    # roofline of the step kernel: algorithmic bytes = 2 * 19 * sizeof(storage) per open node
    alg = 2 * 19 * es * n_open
    peak, peak_kind = peaks()
    achieved = alg / (per_step * 1e-3) / 1e9
    key = f"k_flow_aa_{a.precision}_config2"
    tr = traffic_per_launch(key)
    roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": tr, "peak_source": peak_kind, "algorithmic_bytes_per_launch": alg,
            "kernel": "k_flow_aa (AA even/odd)"}

    # end to end through the C ABI with host buffers: create (material upload) + init (list upload)
    # + the same steps + velocity read back to the host
    D.close()
    del D
    torch.cuda.synchronize()
    k_e2e = a.steps
    t0 = time.perf_counter()
    E = clb.Domain(mat, nx, ny, nz, cfg["tau"], flow_precision=prec, device=local)
    E.flow_init(cfg["delta_p"])
    E.flow_step(k_e2e)
    u = E.velocity()
    t_e2e = time.perf_counter() - t0
    ste = E.flow_stats()
    E.close()
    e2e_val = world * n_open * k_e2e / t_e2e / 1e6
    h2d = nx * ny * nz + 4 * ste["active_nodes"]
    d2h = u.nbytes

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu:
        v, threads, steps, dt = oracle_mlups(mat, cfg["shape"], cfg["tau"], cfg["delta_p"], 12.0, 2, 50)
        cpu = {"value": v, "unit": "MLUPS", "cores": threads, "kind": "port", "cpu": cpu_name(),
               "sample": f"{steps} FP64 steps of the full 258x128x128 map in {dt:.1f} s (OpenMP)"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "MLUPS", "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": a.precision, "data": "synthetic (seeded sphere pack)",
            "config": {"workload": cfg["name"] + f", D3Q19 IncBGK, {a.precision.upper()} populations",
                       "nx": nx, "ny": ny, "nz": nz, "open_voxels": n_open, "active_nodes": n_active,
                       "all_voxel_mlups": all_vox, "l2": "flushed between timed steps (256 MB write); "
                       "compacted lattice %.0f MB" % (19 * es * n_active / 1e6), "parallelism": f"replicas x{world}",
                       "autotune": tuned},
            "roofline": roof,
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_val, "unit": "MLUPS", "h2d_bytes_per_step": h2d / k_e2e,
                    "d2h_bytes_per_step": d2h / k_e2e,
                    "note": "one job through the C ABI: create + init + K steps + velocity to host, wall clock"},
            "gpu_launches": a.steps,
            "clocks": clocks.summary(),
        }
        print(json.dumps(line))
    if world > 1:
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
