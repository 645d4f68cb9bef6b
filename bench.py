#!/usr/bin/env python
"""Throughput of the coupled reactive-transport step on the 256^3 sphere pack (porosity 0.40):
D3Q19 flow (FP32) + 8 D3Q7 species (FP32) with dual-Monod kinetics of two biofilm microbes, the
biofilm automaton every iteration and the flow re-solved every 500 iterations -- the largest
configuration that fits one GPU.

A step is one update interval: 500 coupled iterations (fused transport step of all species,
automaton, dynamics refresh) followed by the flow re-solve to the ValueTracer criterion 1e-6 and
the velocity coupling, driven by clb_run in the reference's loop order. The default 20 steps are
the configuration's 10,000 iterations. MLUPS counts lattice-node updates of both lattices: species
x open voxels per transport iteration plus open voxels per flow iteration. The lattices (about
1.5 GB of species populations) are far larger than L2, so no flush is needed.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Side measurements in the same JSON line (rank 0, one GPU; --no-extra skips them):
  "flow"       the D3Q19 step alone on the 256x128x128 pack (FP32, L2 flushed between steps) and
               its roofline;
  "d3q7"       the fused transport step alone with and without the thermodynamic gate;
  "precision"  FP64 / FP32 / FP16-shifted flow throughput and the velocity, permeability and
               concentration errors of the reduced-precision paths against the FP64 path;
  "speciation" the 5 x 12 tableau in transport: Newton-Raphson against the trained surrogate;
  "ensemble"   96 uneven domains with flow and 3 species advanced by the batched steps.

Multi-GPU: the domain does not shard on this path (single-domain solver); each rank advances
its own replica and the value is the sum over ranks divided by the slowest rank's time.
The reference arm times the FP64 CPU restatement of the reference path (the reference itself
needs Palabos, which is not available) on all host cores, on the full map of the same
configuration, built without the product library.
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
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    p.add_argument("--no-extra", action="store_true", help="skip the D3Q7, precision and speciation legs")
    p.add_argument("--scale", type=float, default=1.0, help="shrink the workload (testing only)")
    p.add_argument("--no-autotune", action="store_true",
                   help="keep the library's default kernel variants (profiling runs: timings under a profiler "
                        "would mislead the autotuner)")
    p.add_argument("--leg", choices=["flow", "d3q7", "precision", "speciation", "ensemble"],
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


class CoupledOracle:
    """The FP64 CPU restatement of the coupled step (oracle/) on a configuration's full map: flow
    lattice, the species lattices with the kinetics, the biofilm automaton. Built from the workload
    description only (maps from the oracle's own generator), so the product library is not loaded."""

    def __init__(self, cfg):
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle

        self.threads = oracle.max_threads()
        oracle.set_threads(self.threads)
        nx, ny, nz = cfg["shape"]
        mat = cfg["mat"]
        self.F = oracle.OracleFlow(mat, nx, ny, nz, cfg["tau"], cfg["delta_p"], bio_codes=cfg["bio_codes"],
                                   perm_ratio=cfg["perm_ratio"])
        self.F.step(2)
        self.A = oracle.OracleAde(mat, nx, ny, nz, cfg["species"], self.F.velocity(), bio_codes=cfg["bio_codes"])
        self.A.set_biomass(cfg["biomass"])
        self.A.set_kinetics(cfg["law"], cfg["params"], cfg["dt"])
        self.A.ca_setup(cfg["bmax"], cfg["biofilm_fraction"], cfg["ca_seed"], bio_codes=cfg["bio_codes"])
        self.S = len(cfg["species"])
        self.n_open = int(np.count_nonzero((mat != 0) & (mat != 1)))
        self.n_flow = self.n_open  # flow BGK nodes: pore and (permeable) biofilm

    def transport_iteration(self):
        """One coupled iteration: the species step with kinetics, then the automaton."""
        t0 = time.perf_counter()
        self.A.step(1)
        self.A.ca_step()
        return time.perf_counter() - t0

    def flow_iteration(self):
        t0 = time.perf_counter()
        self.F.step(1)
        return time.perf_counter() - t0

    def mixed_mlups(self, t_transport, t_flow, flow_per_transport):
        """MLUPS of the coupled step's mix: per transport iteration S x n_open species updates and
        flow_per_transport x n_flow flow updates (the re-solve's iterations spread over its interval)."""
        upd = self.S * self.n_open + flow_per_transport * self.n_flow
        return upd / (t_transport + flow_per_transport * t_flow) / 1e6


def run_reference(a, workloads):
    """The reference arm: the oracle's coupled step on the full map of the headline configuration,
    all host threads, rank 0 only. Each step is one transport iteration (8 species + automaton) and
    one flow iteration, timed separately; the step's MLUPS weights them by the configuration's mix
    (flow iterations of a re-solve over its 500-iteration interval)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    cfg = workloads.pack256cube_8species(scale=a.scale, gen=oracle.sphere_pack)
    t_build = time.perf_counter()
    O = CoupledOracle(cfg)
    t_build = time.perf_counter() - t_build
    mix = workloads.FLOW_PER_TRANSPORT_CONFIG3
    for _ in range(max(1, a.warmup)):
        O.transport_iteration()
        O.flow_iteration()
    tt = tf = 0.0
    for _ in range(a.steps):
        tt += O.transport_iteration()
        tf += O.flow_iteration()
    v = O.mixed_mlups(tt / a.steps, tf / a.steps, mix)
    nx, ny, nz = cfg["shape"]
    sample = (f"{a.steps} coupled iterations (8 species + automaton) and {a.steps} flow iterations of the full "
              f"{nx}x{ny}x{nz} map, FP64, weighted {mix:.3f} flow iterations per transport iteration")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": "MLUPS", "n_gpus": a.gpus, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": (tt + tf) / a.steps * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded sphere pack)",
        "config": {"workload": cfg["name"] + ", coupled step", "nx": nx, "ny": ny, "nz": nz,
                   "open_voxels": O.n_open, "transport_s_per_iteration": tt / a.steps,
                   "flow_s_per_iteration": tf / a.steps, "build_s": t_build},
        "cpu_baseline": {"value": v, "unit": "MLUPS", "cores": O.threads, "kind": "port", "cpu": cpu_name(),
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


def biomass_bytes(bio, open_mask):
    """Biomass bytes per open voxel of one transport step: the 1-byte per-voxel flag; every
    microbe's value read where the flag is set (some microbe holds at least 1e-14); a microbe's
    value written back where it holds biomass (its growth or decay passes the threshold)."""
    b = np.asarray(bio).reshape(len(bio), -1)[:, open_mask.ravel()]
    flag = float(np.mean(np.any(b >= 1e-14, axis=0)))
    held = float(np.sum(np.mean(b >= 1e-14, axis=1)))
    return 1.0 + 8.0 * len(bio) * flag + 8.0 * held, flag


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
    open_mask = (mat != 0) & (mat != 1)
    bio_b, flagged = biomass_bytes([D.biomass(m) for m in range(cfg["biomass"].shape[0])], open_mask)
    # S x 2 x 7 x 4 B populations + 12 B velocity + 1 B material + the biomass bytes
    alg_node = S * 2 * 7 * 4 + 3 * 4 + 1 + bio_b
    achieved = alg_node * n_open / (per * 1e-3) / 1e9
    D.close()
    return {"workload": cfg["name"] + ", FP32 populations, dual-Monod kinetics fused",
            "mlups_d3q7": S * n_open * steps / (ms * 1e-3) / 1e6, "unit": "species x open-voxel updates / s (1e6)",
            "ms_per_step": per, "thermo_gate_ms_per_step": ms_gate / steps, "open_voxels": n_open, "species": S,
            "steps": steps,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "algorithmic_bytes_per_node": alg_node, "biomass_flagged_fraction": flagged,
                         "kernel": "k_ade_aa (all species fused)"}}


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
    """Equilibrium speciation of the 5-component, 12-species tableau inside the transport step of the
    precipitation configuration (192^3 rough fracture, FP32 transport, FP64 speciation, the mineral
    law): Newton-Raphson against the BF16 surrogate. The surrogate is trained on the GPU from
    Newton-Raphson solves of states of this run (1e6 samples of its voxels after 100 coupled steps
    with precipitation, each species scaled by 10^U(-0.6, 0.6)). Timed per transport step with CUDA
    events: speciation off, Newton-Raphson, the surrogate alone (newton_polish 0, every in-range
    answer kept) and the surrogate with a two-step Newton polish and residual check (fallback to
    Newton-Raphson). Errors: relative species difference against Newton-Raphson on 100k held-out
    states drawn like the training set (another seed), for the network alone and polished; and after
    one transport step from the same state (open voxels)."""
    cfg = workloads.fracture192_carbonate(
        lambda nx, ny, nz: clb.geom_generate("fracture", nx, ny, nz, aperture=12.0, roughness=0.3, seed=1004,
                                             walls="none"))
    S, logK, comp = cfg["S"], cfg["logK"], cfg["comp"]
    ns = S.shape[0]
    nx, ny, nz = cfg["shape"]
    mat = cfg["mat"]
    D = clb.Domain(mat, nx, ny, nz, cfg["tau"], flow_precision=clb.F32, ade_precision=clb.F32, device=local)
    stream = torch.cuda.Stream()
    D.set_stream(stream.cuda_stream)
    D.flow_init(cfg["delta_p"])
    D.flow_solve(20000, 1e-6, allow_unconverged=True)
    D.ade_init(cfg["species"])
    D.couple_velocity()
    D.speciation_setup(S, logK, comp, tol=1e-10)
    D.set_speciation_mode(clb.SPEC_NR)
    D.set_abiotic_kinetics(clb.LAW_MINERAL, cfg["mineral"], 0)
    D.set_concentration(cfg["mineral_species"], cfg["deposit"])
    D.precip_setup(cfg["mineral_species"], cfg["full"], seal_flow=1, flow_max_iterations=2000, flow_eps=1e-6)
    sealed = 0
    for _ in range(10):
        D.ade_step(10)
        sealed += D.geometry_update(allow_unconverged=True)[0]
    t_train = time.perf_counter()
    rep = D.surrogate_train([-6.0] * ns, [-2.5] * ns, n_samples=1000000, epochs=60, batch=1024, patience=8,
                            learning_rate=3e-3, seed=1004, from_domain=True, jitter=0.6)
    t_train = time.perf_counter() - t_train
    open_ = (D.material() == 2)
    n_open = int(np.count_nonzero(open_))
    # held-out states: the run's voxel states, jittered like the training set (another seed)
    conc = np.stack([D.concentration(s)[open_] for s in range(ns)], axis=1)
    rng = np.random.default_rng(77)
    pick = rng.choice(conc.shape[0], size=min(100000, conc.shape[0]), replace=False)
    states = np.maximum(conc[pick], 1e-30) * 10.0 ** rng.uniform(-0.6, 0.6, size=(pick.size, ns))
    states = states[(states @ S > 0).all(axis=1)]
    nr, _ = D.speciation_solve(states)
    D.surrogate_set_check(0.02, 0, 1e30)
    raw, acc_raw = D.surrogate_predict(states, residual_check=False)
    D.surrogate_set_check(0.02, 2, 1e-6)
    pol, acc_pol = D.surrogate_predict(states, residual_check=True)
    r_raw = np.abs(raw / nr - 1)[acc_raw]
    r_pol = np.abs(pol / nr - 1)[acc_pol]
    times = {}
    used = {}
    modes = (("off", clb.SPEC_OFF, None), ("nr", clb.SPEC_NR, None), ("raw", clb.SPEC_MLP_NR, (0.02, 0, 1e30)),
             ("polished", clb.SPEC_MLP_NR, (0.02, 2, 1e-6)))
    for key, mode, chk in modes:
        if chk:
            D.surrogate_set_check(*chk)
        D.set_speciation_mode(mode)
        s0 = D.speciation_stats()
        times[key] = timed_steps(torch, stream, D.ade_step, steps, 2) / steps
        s1 = D.speciation_stats()
        used[key] = (s1["surrogate_used"] - s0["surrogate_used"]) / max(1, s1["solves"] - s0["solves"])
    # one transport step from the same state under each mode
    pops0 = [D.ade_populations(s) for s in range(ns)]
    mineral0 = D.concentration(cfg["mineral_species"])
    res = {}
    for key, mode, chk in modes[1:]:
        for s in range(ns):
            D.set_ade_populations(s, pops0[s])
        D.set_concentration(cfg["mineral_species"], mineral0)
        if chk:
            D.surrogate_set_check(*chk)
        D.set_speciation_mode(mode)
        D.ade_step(1)
        res[key] = np.array([D.concentration(s)[open_] for s in range(ns)])
    step_err = {}
    for key in ("raw", "polished"):
        a, b = res[key], res["nr"]
        step_err[key] = float(np.max(np.abs(a / np.where(b == 0, 1, b) - 1)))
    D.close()
    t_nr = times["nr"] - times["off"]
    out = {"workload": cfg["name"] + ", FP32 transport, FP64 speciation", "open_voxels": n_open,
           "voxels_sealed_before_training": sealed, "nr_ms_per_step": t_nr,
           "nr_solves_per_s": n_open / (t_nr * 1e-3)}
    for key in ("raw", "polished"):
        t = times[key] - times["off"]
        r = r_raw if key == "raw" else r_pol
        out[key] = {"ms_per_step": t, "solves_per_s": n_open / (t * 1e-3), "speedup_vs_nr": t_nr / t,
                    "kept_fraction_in_step": used[key],
                    "heldout_max_rel_err": float(r.max()), "heldout_p99_rel_err": float(np.percentile(r, 99)),
                    "heldout_median_rel_err": float(np.median(r)),
                    "heldout_in_range": float((acc_raw if key == "raw" else acc_pol).mean()),
                    "one_step_max_rel_err": step_err[key]}
    out["training"] = {"seconds": t_train, "val_mse": rep["val_mse"], "epochs": rep["epochs"], "steps": rep["steps"],
                       "ms_per_minibatch": t_train * 1e3 / max(1, rep["steps"]), "n_train": rep["n_train"],
                       "source": "states of this run after 100 coupled steps, jitter 0.6 decades"}
    return out


def bench_ensemble(clb, workloads, torch, local, peak, steps=5000):
    """96 independent uneven domains (the parameter-sweep configuration), FP32, each with a D3Q19
    flow and 3 D3Q7 species with Monod kinetics, advanced `steps` steps by the batch after its
    autotuner (persistent item tables against per-lattice launches, the flow step plain or staged),
    timed with CUDA events on the batch's stream. Roofline: algorithmic bytes per step = flow nodes x 2 x 19 x 4 B + transport
    nodes x (3 species x 2 x 7 x 4 B + 3 x 4 B velocity + 1 B material), over the measured copy
    bandwidth. Also timed: the per-lattice schedule with the plain per-node flow step (1000 steps)
    and the domains stepped one after another through their own handles (20 steps)."""
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
    stream = torch.cuda.Stream()
    B = clb.Batch(doms)
    B.set_stream(stream.cuda_stream)
    tuned = B.autotune(16)
    sched = B.get_schedule()
    nf, nt = B.counts()
    step_bytes = nf * 2 * 19 * 4 + nt * (3 * 2 * 7 * 4 + 3 * 4 + 1)
    ms = timed_steps(torch, stream, B.step, steps, 8) / steps
    # the per-lattice schedule with the plain flow step on the same domains
    B.schedule(persistent=False)
    ms_lattice = timed_steps(torch, stream, B.step, 1000, 4) / 1000
    B.schedule(**sched)
    # the same domains one by one (each call enqueues its own launches)
    k = 20
    torch.cuda.synchronize()
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
    achieved = step_bytes / (ms * 1e-3) / 1e9
    return {"workload": cfg["name"] + ", FP32", "domains": n, "flow_nodes": nf, "transport_nodes": nt,
            "steps": steps, "ms_per_step": ms, "domain_steps_per_s": n / (ms * 1e-3),
            "aggregate_mlups": (nf + 3 * nt) / (ms * 1e-3) / 1e6,
            "unit": "domain-steps / s; MLUPS = flow node + species x transport node updates / s (1e6)",
            "schedule": sched, "per_lattice_plain_ms_per_step": ms_lattice,
            "speedup_vs_per_lattice_plain": ms_lattice / ms,
            "one_by_one_ms_per_step": dt1 * 1e3, "speedup_vs_one_by_one": dt1 / (ms * 1e-3),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "bytes_per_step": step_bytes},
            "autotune": tuned,
            "timing": f"CUDA events on the batch stream around {steps} steps (graph-replayed launches); "
                      "one-by-one: host clock, 20 steps"}


def bench_flow(clb, workloads, torch, local, peak, steps=200, warmup=20, precision="f32", autotune=True):
    """The D3Q19 step alone on the 256x128x128 overlapping-sphere pack (porosity 0.35, tau 0.7):
    the compacted FP32 lattice (~113 MB) is about the size of L2, so L2 is flushed between timed
    steps on the same stream (a 256 MB buffer written and then read back, so the L2 holds clean
    lines of that buffer); one event pair per step."""
    cfg = workloads.pack256x128x128()
    prec = {"f64": clb.F64, "f32": clb.F32, "f16s": clb.F16S}[precision]
    es = {"f64": 8, "f32": 4, "f16s": 2}[precision]
    nx, ny, nz = cfg["shape"]
    D = clb.Domain(cfg["mat"], nx, ny, nz, cfg["tau"], flow_precision=prec, device=local)
    stream = torch.cuda.Stream()
    D.set_stream(stream.cuda_stream)
    D.flow_init(cfg["delta_p"])
    tuned = D.autotune(20) if autotune else "defaults"
    st = D.flow_stats()
    n_open = st["bgk_nodes"]
    D.flow_step(warmup)
    D.sync()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    flush_sum = torch.empty((), dtype=torch.int64, device="cuda")
    ev0 = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    ev1 = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    for k in range(steps):
        ev0[k].record(stream)
        D.flow_step(1)
        ev1[k].record(stream)
        with torch.cuda.stream(stream):
            flush.fill_(k & 255)
            torch.sum(flush.view(torch.int64), dim=0, out=flush_sum)
    ev1[-1].synchronize()
    ms = sum(e0.elapsed_time(e1) for e0, e1 in zip(ev0, ev1))
    D.close()
    per = ms / steps
    alg = 2 * 19 * es * n_open
    achieved = alg / (per * 1e-3) / 1e9
    return {"workload": cfg["name"] + f", D3Q19 IncBGK, {precision.upper()} populations",
            "mlups_d3q19": n_open * steps / (ms * 1e-3) / 1e6, "ms_per_step": per, "open_voxels": n_open,
            "autotune": tuned, "l2": "flushed between timed steps (256 MB write, then read back)",
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": traffic_per_launch(f"k_flow_aa_{precision}_pack256x128x128"),
                         "algorithmic_bytes_per_launch": alg, "kernel": step_kernels(tuned, precision)}}


def setup_config3(clb, cfg, local, stream=None, autotune=True, mat=None, biomass=None):
    """The coupled configuration on one device: flow to the ValueTracer criterion from rest, the
    species lattices at rest, the biomass fields, the kinetics, the automaton."""
    nx, ny, nz = cfg["shape"]
    D = clb.Domain(cfg["mat"] if mat is None else mat, nx, ny, nz, cfg["tau"], flow_precision=clb.F32,
                   ade_precision=clb.F32, bio_codes=cfg["bio_codes"], perm_ratio=cfg["perm_ratio"], device=local)
    if stream is not None:
        D.set_stream(stream.cuda_stream)
    D.flow_init(cfg["delta_p"])
    tuned = D.autotune(10) if autotune else "defaults"
    it, conv = D.flow_solve(cfg["flow_max_iterations"], cfg["eps"], allow_unconverged=True)
    D.ade_init(cfg["species"])
    D.couple_velocity()
    D.set_biomass(cfg["biomass"] if biomass is None else biomass)
    D.set_kinetics(cfg["law"], cfg["params"], cfg["dt"])
    D.ca_setup(cfg["bmax"], cfg["biofilm_fraction"], cfg["ca_seed"])
    return D, {"initial_flow_iterations": it, "initial_flow_converged": conv, "autotune": tuned}


def run_block(D, cfg):
    """One step of the headline: one update interval of the coupled step."""
    return D.run(cfg["resolve_every"], ca=True, ade_update_interval=1, resolve_every=cfg["resolve_every"],
                 flow_max_iterations=cfg["flow_max_iterations"], flow_eps=cfg["eps"])


def main():
    a = args_()
    import workloads

    if a.impl == "reference":
        run_reference(a, workloads)
        return

    import clb
    import torch

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    peak, peak_kind = peaks()
    if a.leg:
        fn = {"d3q7": lambda: bench_d3q7(clb, workloads, torch, local, peak, steps=10, warmup=3, scale=a.scale),
              "flow": lambda: bench_flow(clb, workloads, torch, local, peak, autotune=not a.no_autotune),
              "precision": lambda: bench_precision(clb, workloads, torch, local),
              "speciation": lambda: bench_speciation(clb, workloads, torch, local),
              "ensemble": lambda: bench_ensemble(clb, workloads, torch, local, peak)}.get(a.leg)
        if fn is not None:
            print(json.dumps({"leg": a.leg, "scale": a.scale, a.leg: fn()}))
            return
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    cfg = workloads.pack256cube_8species(scale=a.scale)
    nx, ny, nz = cfg["shape"]
    S = len(cfg["species"])
    M = cfg["biomass"].shape[0]
    stream = torch.cuda.Stream()
    # warm-up: W update intervals on one instance (kernels loaded, variants tuned); the timed K
    # intervals are the first K of a fresh instance, the configuration's own iterations 0 .. 500 K,
    # the same work the end-to-end job below does
    W, setup_info = setup_config3(clb, cfg, local, stream, autotune=not a.no_autotune)
    for _ in range(a.warmup):
        run_block(W, cfg)
    W.sync()
    W.close()
    del W
    D, setup_info = setup_config3(clb, cfg, local, stream, autotune=not a.no_autotune)
    n_open = int(np.count_nonzero((cfg["mat"] != 0) & (cfg["mat"] != 1)))
    n_flow = D.flow_stats()["bgk_nodes"]
    D.sync()
    barrier()
    torch.cuda.synchronize()
    reps, ms_blocks = [], []
    # the timed region is an NVTX range ("timed"), so a profiler can take its launches alone
    torch.cuda.nvtx.range_push("timed")
    with ClockSampler(local) as clocks:
        for _ in range(a.steps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            reps.append(run_block(D, cfg))
            e1.record(stream)
            e1.synchronize()
            ms_blocks.append(e0.elapsed_time(e1))
    torch.cuda.nvtx.range_pop()
    torch.cuda.synchronize()
    barrier()
    final = D.reduce()
    D.close()
    del D
    ms = max_over_ranks(torch, sum(ms_blocks), world, "cuda")
    iters = sum(r["iterations"] for r in reps)
    flow_its = sum(r["flow_iterations"] for r in reps)
    upd = S * n_open * iters + n_flow * flow_its
    value = world * upd / (ms * 1e-3) / 1e6
    ms_transport = sum(r["ms_transport"] for r in reps)
    launches = sum(r["launches"] for r in reps)

    # end to end through the C ABI with host buffers: the material map and the biomass fields go in
    # from pinned host memory; create, flow solve from rest, species set-up, the same K update
    # intervals, and every species' concentration and the biomass back into pinned host memory
    t_e2e = None
    job = {}
    if rank == 0 or world > 1:
        mat_host = torch.empty(cfg["mat"].size, dtype=torch.int8, pin_memory=True).numpy()
        mat_host[:] = cfg["mat"]
        bio_host = torch.empty(cfg["biomass"].size, dtype=torch.float64, pin_memory=True).numpy()
        bio_host[:] = cfg["biomass"].ravel()
        out_host = torch.empty((S + M, nx * ny * nz), dtype=torch.float64, pin_memory=True).numpy()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        E, _ = setup_config3(clb, cfg, local, None, autotune=False, mat=mat_host, biomass=bio_host)
        E.sync()
        t1 = time.perf_counter()
        e_reps = [run_block(E, cfg) for _ in range(a.steps)]
        E.sync()
        t2 = time.perf_counter()
        lib = clb.lib()
        for s in range(S):
            E._check(lib.clb_get_field(E.h, clb.FIELD_CONCENTRATION, s, out_host[s].ctypes.data_as(clb.C.c_void_p), 0))
        for m in range(M):
            E._check(lib.clb_get_field(E.h, clb.FIELD_BIOMASS, m, out_host[S + m].ctypes.data_as(clb.C.c_void_p), 0))
        t3 = time.perf_counter()
        E.close()
        t_e2e = t3 - t0
        job = {"setup_s": t1 - t0, "steps_s": t2 - t1, "result_to_host_s": t3 - t2}
        # the job's own updates (the same iterations as the timed region; its re-solves may take
        # a few iterations more or less)
        e_upd = S * n_open * sum(r["iterations"] for r in e_reps) + n_flow * sum(r["flow_iterations"] for r in e_reps)
        e2e_val = world * e_upd / t_e2e / 1e6
        h2d = mat_host.nbytes + bio_host.nbytes
        d2h = out_host.nbytes

    # roofline of the dominant kernel, the fused transport step: algorithmic bytes per open node =
    # S x 2 x 7 x 4 B populations + 12 B velocity + 1 B material + the biomass bytes (flag, reads
    # where it is set, writes where a microbe holds biomass), the mean of the first and last states
    # of the K intervals (the biofilm grows in between)
    # (the last state from the end-to-end job, which runs the same intervals from the same start and
    # reads its biomass back anyway)
    open_mask = (cfg["mat"] != 0) & (cfg["mat"] != 1)
    bio_start = biomass_bytes(cfg["biomass"], open_mask)
    bio_end = biomass_bytes(out_host[S:S + M], open_mask) if t_e2e is not None else bio_start
    alg_node = S * 2 * 7 * 4 + 3 * 4 + 1 + 0.5 * (bio_start[0] + bio_end[0])
    per_launch = ms_transport / max(1, iters)
    achieved = alg_node * n_open / (per_launch * 1e-3) / 1e9
    roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": traffic_per_launch("k_ade_aa_f32_pack256cube_8species"), "peak_source": peak_kind,
            "algorithmic_bytes_per_launch": alg_node * n_open, "algorithmic_bytes_per_node": alg_node,
            "biomass_flagged_fraction": [bio_start[1], bio_end[1]],
            "kernel": "k_ade_aa (all 8 species fused, even/odd AA steps) + k_ade_neumann, the fused transport "
                      "step; mean device time per iteration from CUDA events on the handle's stream",
            "share_of_step": ms_transport / sum(ms_blocks)}

    extra = {}
    if rank == 0 and world == 1 and not a.no_extra and a.scale == 1.0:
        for key, fn in (("flow", lambda: bench_flow(clb, workloads, torch, local, peak, autotune=not a.no_autotune)),
                        ("d3q7", lambda: bench_d3q7(clb, workloads, torch, local, peak)),
                        ("precision", lambda: bench_precision(clb, workloads, torch, local)),
                        ("speciation", lambda: bench_speciation(clb, workloads, torch, local)),
                        ("ensemble", lambda: bench_ensemble(clb, workloads, torch, local, peak))):
            try:
                extra[key] = fn()
            except Exception as exc:  # a failed side measurement must not hide the headline line
                extra[key] = {"error": f"{type(exc).__name__}: {exc}"}
            torch.cuda.synchronize()

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu:
        # the oracle on the full map (its own map generator, the same voxels), a bounded sample:
        # two coupled iterations and two flow iterations, weighted by this run's own mix
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle

        ocfg = workloads.pack256cube_8species(scale=a.scale, gen=oracle.sphere_pack)
        O = CoupledOracle(ocfg)
        O.transport_iteration()
        tt = sum(O.transport_iteration() for _ in range(2)) / 2
        tf = sum(O.flow_iteration() for _ in range(2)) / 2
        mix = flow_its / max(1, iters)
        cpu = {"value": O.mixed_mlups(tt, tf, mix), "unit": "MLUPS", "cores": O.threads, "kind": "port",
               "cpu": cpu_name(),
               "sample": f"2 coupled iterations (8 species + automaton, {tt:.2f} s each) and 2 flow iterations "
                         f"({tf:.2f} s each) of the full map, FP64, weighted by this run's {mix:.3f} flow "
                         "iterations per transport iteration"}
        # the same code on one thread: one coupled and one flow iteration
        oracle.set_threads(1)
        t1 = O.transport_iteration()
        f1 = O.flow_iteration()
        cpu["single_thread"] = {"value": O.mixed_mlups(t1, f1, mix), "unit": "MLUPS", "cores": 1,
                                "sample": f"1 coupled iteration ({t1:.2f} s) and 1 flow iteration ({f1:.2f} s) of "
                                          "the full map, weighted the same way"}
        del O

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "MLUPS", "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": ms / a.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded sphere pack)",
            "config": {"workload": cfg["name"] + ", coupled step: FP32 D3Q19 flow + 8 x FP32 D3Q7, dual-Monod, "
                       "biofilm automaton every iteration, flow re-solved every 500 iterations",
                       "step": "one update interval = 500 coupled iterations + the flow re-solve (1e-6)",
                       "timed": "update intervals 1..K of a fresh instance (after W warm-up intervals on another)",
                       "nx": nx, "ny": ny, "nz": nz, "species": S, "microbes": M, "open_voxels": n_open,
                       "flow_nodes": n_flow, "iterations": iters, "flow_iterations": flow_its,
                       "ca_sweeps": sum(r["ca_sweeps"] for r in reps),
                       "mask_changes": sum(r["mask_changes"] for r in reps),
                       "ms_transport": ms_transport, "ms_ca": sum(r["ms_ca"] for r in reps),
                       "ms_flow": sum(r["ms_flow"] for r in reps),
                       "l2": "not flushed: 1.5 GB of species populations per step, far larger than L2",
                       "parallelism": f"replicas x{world}", "final_totals": list(map(float, final["total"])),
                       "final_biomass": list(map(float, final["biomass"][:M])), **setup_info},
            "roofline": roof,
            "cpu_baseline": cpu,
            "e2e": None if t_e2e is None else {
                "value": e2e_val, "unit": "MLUPS", "h2d_bytes_per_step": h2d / a.steps,
                "d2h_bytes_per_step": d2h / a.steps,
                "note": "one job through the C ABI: create from pinned host buffers, flow solve from rest, "
                        "species set-up, the same K update intervals as the timed region, every concentration "
                        "and biomass field to pinned host memory; wall clock", "job_phases_s": job},
            "gpu_launches": launches,
            "clocks": clocks.summary(),
        }
        line.update(extra)
        print(json.dumps(line))
    if world > 1:
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
