"""Benchmark: Biot-Savart node velocities per second at a 1e-5 relative-error target, tuned FP32
(learned parameters) against plain FP64, on the 1M-node tangle.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload NAME]

One step = one velocity evaluation on all nodes of the workload: device-side point data
(quintic splines, quadrature points), cell lists, pair kernel, local term, NUFFT long range.
The headline `value` is the tuned form: mixed precision at the Ewald/NUFFT parameters the
learned predictor chooses for the target (checked against a plain FP64 evaluation); the plain
FP64 and mixed forms at the workload's own parameters are reported under `forms`.  `value` is
measured with the filament nodes already resident in HBM; `e2e` goes through the public API
(velocity_on_nodes_ with host arrays): host->device copy of the nodes and device->host copy of
the velocities inside the timed region.  Multi-GPU (torchrun): every rank evaluates its own
independent tangle (weak scaling, no collective on the data path).
"""

from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

# Hardware work queues of this process's CUDA context (read when the context is created, so set before
# any CUDA call): the batching form runs one stream per system, and with the default 8 queues streams
# share queues and their kernels run one after another.
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "Biot–Savart node-velocities/s at 1e-5 rel err: tuned FP32 vs plain FP64 GPU"
UNIT = "node-velocities/s"
F_PAIR_VEL = 40.0  # flops per in-range pair (velocity), convention of the roofline model
L2_FLUSH_BYTES = 256 << 20
L2_BYTES = 126e6  # B200 L2 cache


def load_package():
    import importlib.util
    name = "vortexpasta_b200"
    if name in sys.modules:
        return sys.modules[name]
    pkg = ROOT / "vortexpasta.jl_b200"
    spec = importlib.util.spec_from_file_location(name, pkg / "__init__.py", submodule_search_locations=[str(pkg)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


WORKLOAD_DESC = {
    "tangle20k": "tangle20k: 100 random perturbed rings x 200 nodes = 20,000 nodes, L=2pi, quintic splines, GL(3), "
                 "beta=3.5, r_cut=L/8 (alpha=4.456), Ns=128 (FFT 192^3), sigma=1.5, m=4, Gamma=1, a=1e-8, "
                 "Delta=1/4, CellLists M=2",
    "ring64": "ring64: single ring R=L/4, 64 nodes, beta=3.5, r_cut=L/4, Ns=32 (FFT 48^3), m=4",
    "tangle1m": "tangle1m: 5000 rings x 200 nodes = 1,000,000 nodes, beta=4, r_cut=L/16, Ns=512 (FFT 768^3), m=5",
}


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)), int(os.environ.get("WORLD_SIZE", 1))


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def __enter__(self):
        import tempfile
        self.path = tempfile.mktemp(suffix=".csv")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.proc or not self.path or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_oracle_time(fs, p, nthreads, reps):
    """Oracle (CPU FP64 restatement) timing: returns (seconds per evaluation, velocity)."""
    from oracle import oracle as O
    v = None
    ts = []
    for _ in range(reps):
        t0 = time.perf_counter()
        v, _, _ = O.compute_on_nodes(p, fs, velocity=True, streamfunction=False, nthreads=nthreads)
        ts.append(time.perf_counter() - t0)
    return min(ts), v


def host_cores():
    return len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()


def run_reference(args):
    rank, _, world = dist_env()
    if rank != 0:
        return 0
    vp = load_package()
    fs, p, desc = cpu_sample(vp, args.workload)
    Np = sum(len(f) for f in fs)
    cores = host_cores()
    for _ in range(min(args.warmup, 1)):
        cpu_oracle_time(fs, p, cores, 1)
    times = [cpu_oracle_time(fs, p, cores, 1)[0] for _ in range(args.steps)]
    t = statistics.mean(times)
    value = Np / t
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * t, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD_DESC[args.workload], "fields": "velocity"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": f"one evaluation per step; {desc}"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def stage_model(stage, S):
    """Algorithmic work per launch of each stage: (bound, amount, unit).  S["gsz"] is the grid
    element size (8 bytes in the plain form, 4 in the FP32 forms)."""
    Np, Nq, n3, nc3, g = S["Np"], S["Nq"], S["n3"], S["nc3"], S["gsz"]
    if stage == "pairs":
        return S["pair_bound"], S["pairs"] * F_PAIR_VEL, "flop"
    if stage == "spread":
        return "hbm", Nq * 6 * 8 + 3 * n3 * g, "byte"
    if stage == "interp":
        return "hbm", 3 * n3 * g + Np * 3 * 8 + Np * 3 * 8, "byte"
    if stage == "fourier":
        # reads the retained modes of the forward transform, writes the whole (zero-padded) grid
        # for the inverse transform and the FP64 vorticity coefficients
        return "hbm", 3 * S["nm"] * 2 * g + 3 * nc3 * 2 * g + 3 * S["nm"] * 16, "byte"
    if stage in ("fft_forward", "fft_inverse"):
        return "hbm", 2 * 2 * 3 * n3 * g, "byte"
    if stage == "local_self":
        # per node: position, previous index, s', s'', delta^-, delta^+, output read + write; each
        # quadrature point (position + charge) is gathered by the two nodes of its segment but
        # counted once
        return "hbm", Np * (3 * 8 + 4 + 6 * 8 + 2 * 8 + 2 * 3 * 8) + Nq * 6 * 8, "byte"
    if stage == "geometry":
        return "hbm", Np * 3 * 8 + Np * (3 * 3 * 8 + 12 * 8) + Np * (11 * 8) + Nq * 6 * 8, "byte"
    if stage == "cell_lists":
        return "hbm", Nq * (6 * 8 * 3 + 4 * 4) + Np * 16, "byte"
    return "hbm", 0.0, "byte"


def read_traffic(kernel_stage, workload, form):
    """DRAM bytes per launch of a stage's kernel from the committed ncu-derived table for this
    workload and form (profiles/dram_traffic_<workload>_<form>.txt), if present."""
    f = ROOT / "profiles" / f"dram_traffic_{workload}_{form}.txt"
    if not f.exists():
        return None
    for line in f.read_text().splitlines():
        parts = line.split()
        if len(parts) >= 2 and not parts[0].startswith("#") and parts[0] == kernel_stage:
            try:
                return float(parts[1])
            except ValueError:
                return None
    return None


def rank_workload(vp, workload: str, rank: int):
    """Each rank evaluates its own independent system (weak scaling): same generator and
    parameters, seed 42 + rank."""
    if workload == "ring64":
        return vp.configs.ring64()
    return vp.configs.WORKLOADS[workload](seed=42 + rank)


def max_over_ranks(values, device, world):
    """Element-wise max over ranks of per-rank timings (the job's time is its slowest rank)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor(values, dtype=torch.float64, device=device)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.tolist()


def measure_form(vp, p, fs, args, dev, world, local_rank):
    """Time one arithmetic form: device-resident steps (with per-stage events) and end-to-end
    steps through velocity_on_nodes_.  Returns per-rank-max timings and the velocities."""
    import torch
    import torch.distributed as dist
    from vortexpasta_b200 import _lib
    nodes, offsets = vp.curves.concat(fs)
    stream = torch.cuda.Stream(device=dev)
    cache = vp.init_cache(p)
    cache.set_stream(stream.cuda_stream)
    nodes_dev = torch.from_numpy(nodes).to(dev)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)
    torch.cuda.synchronize()

    def step_device():
        cache.set_filaments(None, on_device_ptr=nodes_dev.data_ptr(), offsets=offsets)
        cache.compute(_lib.VELOCITY)

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            step_device()
    torch.cuda.synchronize()

    # ---- timed region: device-resident inputs ----
    launches0 = cache.launch_count()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local_rank) as clk:
        with torch.cuda.stream(stream):
            for k in range(args.steps):
                flush.zero_()  # L2 flush between timed steps (outside the events)
                starts[k].record(stream)
                step_device()
                ends[k].record(stream)
        torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    launches = cache.launch_count() - launches0
    step_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]

    # ---- per-stage breakdown (untimed steps; stage timing runs the stages one after another) ----
    cache.stage_timing(True)
    stage_ms = {}
    with torch.cuda.stream(stream):
        for k in range(min(args.steps, 3)):
            flush.zero_()
            step_device()
            for name, ms in cache.stage_times().items():
                stage_ms.setdefault(name, []).append(ms)
    torch.cuda.synchronize()
    cache.stage_timing(False)
    total_ms = sum(step_ms)
    pairs_in_range, _ = cache.pair_counts()
    v_dev = cache.get(_lib.VELOCITY)

    # ---- e2e: the flat host-buffer C-ABI calls (vpbs_set_filaments with host nodes, vpbs_compute,
    # vpbs_get into a host array): host->device and device->host copies inside the timed region ----
    v_api = np.zeros((len(nodes), 3))

    def step_e2e():
        cache.set_filaments_flat(nodes, offsets)
        cache.compute(_lib.VELOCITY)
        cache.get(_lib.VELOCITY, v_api)

    with torch.cuda.stream(stream):
        step_e2e()  # warm
        e_starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        e_ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        for k in range(args.steps):
            flush.zero_()
            e_starts[k].record(stream)
            step_e2e()
            e_ends[k].record(stream)
    torch.cuda.synchronize()
    e2e_ms = sum(s.elapsed_time(e) for s, e in zip(e_starts, e_ends))

    cache.close()
    total_ms, e2e_ms = max_over_ranks([total_ms, e2e_ms], dev, world)
    return {"total_ms": total_ms, "e2e_ms": e2e_ms, "stage_ms": stage_ms, "launches": launches,
            "pairs_in_range": pairs_in_range, "v": v_dev.copy(), "v_api": v_api, "clk": clk}


def form_summary(p, m, Np, Nq, world, args, peaks):
    """Throughputs and the per-stage roofline of one measured form (rank 0)."""
    from vortexpasta_b200 import _lib
    n = [_lib.load().vpbs_fft_size(N, p.backend_long.sigma) for N in p.splitting.Ns]
    fp32 = p.precision == "mixed"
    Ns = p.splitting.Ns
    S = {"Np": Np, "Nq": Nq, "n3": n[0] * n[1] * n[2], "nc3": (n[0] // 2 + 1) * n[1] * n[2],
         "nm": (Ns[0] // 2 + 1) * Ns[1] * Ns[2],
         "pairs": m["pairs_in_range"], "nq": len(p.quadrature), "gsz": 4 if fp32 else 8,
         "pair_bound": "fp32" if fp32 else "fp64"}
    avg = {k: statistics.mean(v) for k, v in m["stage_ms"].items()}
    stages = {}
    for name, ms in avg.items():
        bound, amount, unit = stage_model(name, S)
        if ms <= 0:
            continue
        if bound in ("fp64", "fp32"):
            ach = amount / (ms * 1e-3) / 1e12
            pk = peaks[bound]
            stages[name] = {"ms": ms, "bound": bound, "achieved": ach, "unit": "TFLOP/s", "peak": pk,
                            "frac": ach / pk if pk else None}
        else:
            ach = amount / (ms * 1e-3) / 1e9
            stages[name] = {"ms": ms, "bound": "hbm", "achieved": ach, "unit": "GB/s", "peak": peaks["hbm"],
                            "frac": ach / peaks["hbm"]}
            if amount < 2 * L2_BYTES:
                # the stage's algorithmic bytes are within twice the L2 (126 MB): much of its
                # traffic is served from L2, so a fraction of the HBM peak means nothing
                stages[name]["frac"] = None
                stages[name]["note"] = "working set within 2x L2; no HBM fraction"
    if "spread" in stages:
        # grid-value updates of the spreading, Nq (2m)^3 x 3 components (its on-chip work; the HBM
        # figure above counts only the points read and the grid written once)
        stages["spread"]["grid_updates_per_s"] = Nq * (2 * p.backend_long.m) ** 3 * 3 / (stages["spread"]["ms"] * 1e-3)
    dom = max(avg, key=avg.get)
    return {"value": world * Np * args.steps / (m["total_ms"] * 1e-3), "ms_per_step": m["total_ms"] / args.steps,
            "e2e_value": world * Np * args.steps / (m["e2e_ms"] * 1e-3), "stages": stages, "dominant": dom,
            "fft": n[0], "pairs_in_range": int(m["pairs_in_range"])}


def device_peaks(local_rank):
    import ctypes as ct
    from vortexpasta_b200 import _lib
    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
    out = {"hbm": peaks.get("hbm_gbs") or 6650.0,
           "hbm_source": "measured (MEASURED_PEAKS.json hbm_gbs)" if peaks.get("hbm_gbs") else "fallback 6650 GB/s"}
    for key, fp64 in (("fp64", 1), ("fp32", 0)):
        v = ct.c_double()
        out[key] = v.value if _lib.load().vpbs_fma_throughput(local_rank, fp64, ct.byref(v)) == 0 else None
    return out


def errors_vs(v, vref):
    return {"rel_l2_vs_fp64": float(np.linalg.norm(v - vref) / np.linalg.norm(vref)),
            "max_err_vs_fp64": float(np.abs(v - vref).max() / np.abs(vref).max())}


def ensemble_systems(vp, nsys=64, seed=64):
    """The batching-form ensemble: `nsys` random tangles (200-node rings) with node counts
    log-uniform in [2k, 200k], grid Ns = nearest power of two to N^(1/3) * 4 clamped to [64, 256],
    beta = 3.5 (alpha and r_cut from the reference's rule), mixed precision.  Time step:
    min(1e-3 L^2 / Gamma, Kelvin-wave period of the shortest segment) -- the fixed 1e-3 L^2/Gamma
    alone is ~650x above that stability limit and the tangles blow up within a few steps."""
    from vortexpasta_b200.params import (GaussianSplitting, GaussLegendre, NonuniformFFTsBackend, ParamsBiotSavart,
                                         kelvin_wave_period)
    L = 2 * math.pi
    rng = np.random.default_rng(seed)
    out = []
    for k in range(nsys):
        N = 10 ** rng.uniform(math.log10(2000), math.log10(200000))
        nrings = max(10, int(round(N / 200)))
        fs = vp.curves.random_tangle(nrings, 200, L=L, seed=int(rng.integers(1 << 31)))
        Ns = int(min(256, max(64, 2 ** round(math.log2(N ** (1 / 3) * 4)))))
        p = ParamsBiotSavart(Gamma=1.0, a=1e-8, Delta=0.25, splitting=GaussianSplitting(Ls=L, beta=3.5, Ns=Ns),
                             quadrature=GaussLegendre(3), backend_long=NonuniformFFTsBackend(1.5, 4), precision="mixed")
        dmin = min(float(np.linalg.norm(np.roll(f, -1, axis=0) - f, axis=1).min()) for f in fs)
        dt = min(1e-3 * L ** 2 / 1.0, kelvin_wave_period(dmin, a=1e-8, Delta=0.25, Gamma=1.0))
        out.append((fs, p, dt))
    return out


def small_ensemble_systems(vp, nsys=256, seed=65):
    """A launch-bound ensemble: `nsys` small random tangles (5-10 rings x 200 nodes), Ns = 32 (FFT 48^3),
    beta = 3.5, NUFFT m = 4, mixed precision, dt as in ``ensemble_systems``.  Each system's kernels are
    a few microseconds long, so issuing them one by one from the host costs more than running them."""
    from vortexpasta_b200.params import (GaussianSplitting, GaussLegendre, NonuniformFFTsBackend, ParamsBiotSavart,
                                         kelvin_wave_period)
    L = 2 * math.pi
    rng = np.random.default_rng(seed)
    out = []
    for k in range(nsys):
        fs = vp.curves.random_tangle(int(rng.integers(5, 11)), 200, L=L, seed=int(rng.integers(1 << 31)))
        p = ParamsBiotSavart(Gamma=1.0, a=1e-8, Delta=0.25, splitting=GaussianSplitting(Ls=L, beta=3.5, Ns=32),
                             quadrature=GaussLegendre(3), backend_long=NonuniformFFTsBackend(1.5, 4), precision="mixed")
        dmin = min(float(np.linalg.norm(np.roll(f, -1, axis=0) - f, axis=1).min()) for f in fs)
        dt = min(1e-3 * L ** 2 / 1.0, kelvin_wave_period(dmin, a=1e-8, Delta=0.25, Gamma=1.0))
        out.append((fs, p, dt))
    return out


def time_ensemble(vp, all_systems, args, local_rank, rank, world, autotune):
    """RK4 steps of an ensemble replayed as one CUDA graph per step, against the same steps issued
    system by system without a graph (each system on its own streams, so those calls overlap on the
    device too).  With several ranks the systems are sharded by estimated cost
    (timestepping.shard_systems; no data exchange) and the job's time is the max over ranks."""
    import torch
    from vortexpasta_b200 import timestepping, tuning
    L = 2 * math.pi
    costs = [timestepping.system_cost(sum(len(f) for f in fs), tuning.fft_size(p.splitting.Ns[0], p.backend_long.sigma))
             for fs, p, _ in all_systems]
    mine = timestepping.shard_systems(costs, world)[rank]
    systems = [all_systems[i] for i in mine]
    nodes_all = sum(sum(len(f) for f in fs) for fs, _, _ in all_systems)
    nodes = sum(sum(len(f) for f in fs) for fs, _, _ in systems)
    t0 = time.perf_counter()
    ens = timestepping.Ensemble([(fs, p.with_(device=local_rank), dt) for fs, p, dt in systems], device=local_rank,
                                autotune_pairs=autotune)
    t_setup = time.perf_counter() - t0
    try:
        stream = torch.cuda.ExternalStream(ens.stream(), device=local_rank)
        ens.step(2)  # warm-up replays
        ens.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ens.step(args.ensemble_steps)
        e1.record(stream)
        ens.synchronize()
        ms_graph = e0.elapsed_time(e1)
        # the same steps, system by system, no graph (host wall clock around a synchronised loop);
        # `host_ms` is the time the host spends issuing them (the calls return before the device is done)
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        for _ in range(args.ensemble_steps):
            for c, x, (_, _, dt) in zip(ens.caches, ens.nodes, systems):
                timestepping.rk4_step(c, x.data_ptr(), dt)
        host_ms = (time.perf_counter() - t1) * 1e3
        torch.cuda.synchronize()
        ms_seq = (time.perf_counter() - t1) * 1e3
        finite = all(bool(torch.isfinite(x).all()) for x in ens.nodes)
    finally:
        ens.close()
    ms_graph, ms_seq, host_ms, nonfinite = max_over_ranks([ms_graph, ms_seq, host_ms, 0.0 if finite else 1.0],
                                                          local_rank, world)
    evals = 4 * nodes_all * args.ensemble_steps
    kw_limited = sum(1 for _, _, dt in all_systems if dt < 1e-3 * L ** 2)
    out = {"systems": len(all_systems), "nodes_total": nodes_all, "rk4_steps": args.ensemble_steps,
           "ranks": world, "systems_on_rank0": len(systems), "nodes_on_rank0": nodes,
           "node_velocities_per_s": evals / (ms_graph * 1e-3), "ms_per_step": ms_graph / args.ensemble_steps,
           "sequential_node_velocities_per_s": evals / (ms_seq * 1e-3), "graph_speedup": ms_seq / ms_graph,
           "sequential_host_issue_ms_per_step": host_ms / args.ensemble_steps,
           "sequential_ms_per_step": ms_seq / args.ensemble_steps,
           "dt_rule": "min(1e-3 L^2/Gamma, Kelvin-wave period of the shortest segment)",
           "dt_kelvin_wave_limited_systems": kw_limited,
           "setup_s": t_setup, "finite": nonfinite == 0.0}
    if autotune:
        out["autotuned"] = {"pair_block_systems_off_rule": sum(1 for t in ens.tuned if t),
                            "pair_block_edges": sorted(set(ens.tuned)),
                            "spread_mode_systems_cuda_cores": sum(1 for m in ens.spread_modes if m)}
    return out


def measure_ensemble(vp, args, local_rank, rank=0, world=1):
    """The batching form on two ensembles: the 64 random tangles of ``ensemble_systems`` (device-bound:
    the host issues a step's kernels faster than the device runs them, so the graph has nothing to
    save) and the 256 small tangles of ``small_ensemble_systems`` (launch-bound)."""
    big = time_ensemble(vp, ensemble_systems(vp), args, local_rank, rank, world, autotune=True)
    big["description"] = ("64 random tangles, N log-uniform in [2k, 200k] (200-node rings), Ns = nearest power of "
                          "two to N^(1/3)*4 in [64, 256], beta = 3.5, mixed precision, RK4 with dt = min(1e-3 L^2/Gamma, "
                          "Kelvin-wave period of the shortest segment); one CUDA graph launch per RK4 step (all "
                          "systems, one stream each), vs the same steps issued system by system")
    small = time_ensemble(vp, small_ensemble_systems(vp), args, local_rank, rank, world, autotune=True)
    small["description"] = ("256 random tangles of 5-10 rings x 200 nodes, Ns = 32 (FFT 48^3), beta = 3.5, m = 4, "
                            "mixed precision, dt as above; one CUDA graph launch per RK4 step vs the same steps "
                            "issued system by system")
    big["small_systems"] = small
    return big


def run_ours(args):
    import torch
    import torch.distributed as dist
    rank, local_rank, world = dist_env()
    if world > 1:
        dist.init_process_group("nccl" if torch.cuda.is_available() else "gloo",
                                timeout=__import__("datetime").timedelta(seconds=120))
    if not torch.cuda.is_available():
        raise RuntimeError("bench.py needs a CUDA GPU")
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    vp = load_package()
    from vortexpasta_b200 import learned
    fs, p = rank_workload(vp, args.workload, rank)
    p = p.with_(device=local_rank)
    L = p.splitting.Ls[0]
    Np = sum(len(f) for f in fs)
    Nq = Np * len(p.quadrature)
    nodes, offsets = vp.curves.concat(fs)

    # plain FP64 and mixed forms at the workload's parameters
    m64 = measure_form(vp, p, fs, args, dev, world, local_rank)
    mixed = measure_form(vp, p.with_(precision="mixed"), fs, args, dev, world, local_rank) if args.mixed else None
    # tuned form: parameters from the learned predictor (checked against a plain FP64 evaluation,
    # default rule on a miss), FP32 bulk arithmetic
    tuned = tuned64 = None
    if args.tuned:
        choices = learned.ChoiceCache()
        t0 = time.perf_counter()
        choice, info = learned.choose_parameters(fs, L, rtol=args.rtol, device=local_rank, cache=choices)
        t_choose = time.perf_counter() - t0
        # the same configuration class again (a later solve of the same simulation): served by the cache
        t0 = time.perf_counter()
        choice_again, info_again = learned.choose_parameters(fs, L, rtol=args.rtol, device=local_rank, cache=choices)
        t_cached = time.perf_counter() - t0
        assert info_again["cached"] and choice_again == choice
        pt = choice.params(L, "mixed", device=local_rank)
        tuned = measure_form(vp, pt, fs, args, dev, world, local_rank)
        # FP64 at the tuned parameters: separates the gain of the parameter choice from that of
        # the FP32 arithmetic
        tuned64 = measure_form(vp, pt.with_(precision="fp64"), fs, args, dev, world, local_rank) if args.mixed else None
    head = tuned if tuned is not None else m64
    head_p = pt if tuned is not None else p
    # every rank steps its shard of the ensemble (the timing reduction inside is a collective)
    ensemble = measure_ensemble(vp, args, local_rank, rank, world) if args.ensemble_steps > 0 else None

    if rank == 0:
        peaks = device_peaks(local_rank)
        f64 = form_summary(p, m64, Np, Nq, world, args, peaks)
        fh = form_summary(head_p, head, Np, Nq, world, args, peaks)
        d = fh["stages"][fh["dominant"]]
        roof = {"kernel": fh["dominant"], "bound": d["bound"], "achieved": d["achieved"], "peak": d["peak"],
                "unit": d["unit"], "frac": d["frac"],
                "traffic": read_traffic(fh["dominant"], args.workload, "tuned" if tuned is not None else "fp64"),
                "peak_source": {"fp64": "measured FP64 FMA throughput (vpbs_fma_throughput)",
                                "fp32": "measured FP32 FMA throughput (vpbs_fma_throughput)"}.get(d["bound"],
                                                                                                   peaks["hbm_source"])}
        forms = {"fp64": {**{k: f64[k] for k in ("value", "ms_per_step", "e2e_value")},
                          "stages_ms": {k: v["ms"] for k, v in f64["stages"].items()},
                          "description": "plain FP64 at the workload's parameters"}}
        if mixed is not None:
            fm = form_summary(p.with_(precision="mixed"), mixed, Np, Nq, world, args, peaks)
            forms["mixed"] = {**{k: fm[k] for k in ("value", "ms_per_step", "e2e_value")},
                              "speedup_vs_fp64": fm["value"] / f64["value"], **errors_vs(mixed["v"], m64["v"]),
                              "stages_ms": {k: v["ms"] for k, v in fm["stages"].items()},
                              "description": "FP32 pair sum / spreading / FFT / interpolation at the workload's "
                                             "parameters; FP64 positions, separations, local and self terms, "
                                             "accumulation"}
        if tuned is not None:
            forms["tuned"] = {**{k: fh[k] for k in ("value", "ms_per_step", "e2e_value")},
                              "speedup_vs_fp64": fh["value"] / f64["value"],
                              "e2e_speedup_vs_fp64": fh["e2e_value"] / f64["e2e_value"],
                              **errors_vs(tuned["v"], m64["v"]),
                              "parameters": {**choice.as_dict(), "fft": fh["fft"], "rcut_over_L": choice.rcut / L,
                                             "beta": choice.beta_short},
                              "predictor": {"fallback_to_default_rule": bool(info["fallback"]),
                                            "checked_rel_l2": info.get("rel_l2"), "rtol": args.rtol,
                                            "seconds": t_choose, "seconds_cached": t_cached,
                                            "candidates": [{k: a[k] for k in ("rel_l2", "ms", "sigma", "m", "fft") if k in a} |
                                                           {"splitting": a.get("splitting", "gaussian")}
                                                           for a in info["attempts"]]},
                              "stages_ms": {k: v["ms"] for k, v in fh["stages"].items()},
                              "description": ("mixed precision at the cut-off and NUFFT predicted by the learned MLP; "
                                              "Gaussian or Kaiser-Bessel split, whichever met the tolerance in less "
                                              "time in the FP64-checked trial")}
            if tuned64 is not None:
                ft = form_summary(pt.with_(precision="fp64"), tuned64, Np, Nq, world, args, peaks)
                forms["fp64_tuned"] = {**{k: ft[k] for k in ("value", "ms_per_step", "e2e_value")},
                                       "speedup_vs_fp64": ft["value"] / f64["value"],
                                       **errors_vs(tuned64["v"], m64["v"]),
                                       "stages_ms": {k: v["ms"] for k, v in ft["stages"].items()},
                                       "description": "plain FP64 arithmetic at the tuned form's parameters"}
        line = {
            "metric": METRIC, "value": fh["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": fh["ms_per_step"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32" if tuned is not None else "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD_DESC[args.workload],
                       "form": ("tuned FP32 (learned parameters; FP64 positions, separations, local term and "
                                "accumulation), compared with plain FP64 at the workload's parameters under 'forms'"
                                if tuned is not None else "plain FP64"),
                       "fields": "velocity", "target_rel_l2": args.rtol,
                       "parallelism": f"replicas x{world} (independent tangles, no collective)",
                       "l2": "flushed between timed steps (256 MiB write, outside the timed events)"},
            "roofline": roof,
            "stages": fh["stages"],
            "forms": forms,
            "e2e": {"value": fh["e2e_value"], "unit": UNIT, "h2d_bytes_per_step": int(nodes.nbytes + offsets.nbytes),
                    "d2h_bytes_per_step": int(Np * 3 * 8)},
            "gpu_launches": int(head["launches"]),
            "clocks": head["clk"].summary(),
            "pairs_in_range": fh["pairs_in_range"],
        }
        if ensemble is not None:
            line["ensemble"] = ensemble
        if world == 1 and not args.no_cpu_baseline:
            cores = host_cores()
            sfs, sp, desc = cpu_sample(vp, args.workload)
            t_cpu, v_cpu = cpu_oracle_time(sfs, sp, cores, args.cpu_reps)
            line["cpu_baseline"] = {"value": sum(len(f) for f in sfs) / t_cpu, "unit": UNIT, "cores": cores,
                                    "kind": "port", "sample": desc}
            line["accuracy"] = sample_accuracy(vp, args, sfs, sp, v_cpu, pt if tuned is not None else None,
                                               local_rank)
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


def sample_velocity(vp, p, fs):
    """Node velocities of one evaluation of `fs` with parameters `p` (host copy)."""
    from vortexpasta_b200 import _lib
    c = vp.init_cache(p)
    try:
        c.set_filaments(fs)
        c.compute(_lib.VELOCITY)
        return c.get(_lib.VELOCITY)
    finally:
        c.close()


def sample_accuracy(vp, args, sfs, sp, v_oracle, p_tuned, device):
    """Relative L2 errors against the FP64 oracle on the CPU sample of the workload (for tangle1m
    the 1/64-volume sample, with every parameter set carried over at the same absolute cut-off,
    splitting parameter and grid spacing): the plain FP64 and mixed forms at the workload's
    parameters, and the tuned form at its chosen parameters -- the metric's accuracy condition."""
    def rel(v):
        return float(np.linalg.norm(v - v_oracle) / np.linalg.norm(v_oracle))
    sp = sp.with_(device=device)
    out = {"sample": "the cpu_baseline sample; oracle = FP64 CPU restatement at the workload's parameters",
           "fp64_rel_l2_vs_oracle": rel(sample_velocity(vp, sp, sfs))}
    if args.mixed:
        out["mixed_rel_l2_vs_oracle"] = rel(sample_velocity(vp, sp.with_(precision="mixed"), sfs))
    if p_tuned is not None:
        k = SAMPLE_K[args.workload]
        pts = (vp.configs.sample_params(p_tuned, k) if k > 1 else p_tuned).with_(device=device)
        out["tuned_rel_l2_vs_oracle"] = rel(sample_velocity(vp, pts, sfs))
        out["tuned_fp64_rel_l2_vs_oracle"] = rel(sample_velocity(vp, pts.with_(precision="fp64"), sfs))
        out["tuned_meets_target"] = out["tuned_rel_l2_vs_oracle"] <= args.rtol
    return out


SAMPLE_K = {"tangle1m": 4, "tangle20k": 1, "ring64": 1}  # CPU sample = cube of side L / k


def cpu_sample(vp, workload):
    """The bounded CPU sample of a workload: (filaments, parameters, description)."""
    if workload == "tangle1m":
        fs, p = vp.configs.tangle1m_cpu_sample()
        return fs, p, ("tangle1m_cpu_sample: 1/64-volume replica of tangle1m (cube L/4, 78 rings x 200 nodes = "
                       "15,600 nodes, same node density, same absolute r_cut, alpha and grid spacing), "
                       "best of the timed full velocity evaluations (CPU FP64 restatement, OpenMP)")
    fs, p = vp.configs.WORKLOADS[workload]()
    return fs, p, (f"full velocity evaluations of {workload}, best taken (CPU FP64 restatement, OpenMP)")


KERNEL_CASES = {
    "pairs1m": "pair kernel of tangle1m (r_cut = L/16, beta = 4) with a 64^3 Fourier grid, FP64 then mixed",
    "tuned500k": "2500 rings x 200 nodes (500k nodes) at the tuned 1M parameters (alpha = 22.03, r_cut = 0.1561, "
                 "Ns = 341, sigma = 1.5, m = 3), mixed precision",
    "tuned1m": "tangle1m at the Kaiser-Bessel split the tuned form picks (beta = 12.44 from rtol 1e-5 / 4, "
               "r_cut = 0.13956 = L/45, Ns = 192, FFT 288^3, sigma = 1.5, m = 3), mixed precision",
}


def run_kernel_case(args):
    """Small fixed workloads for kernel profiling (three evaluations each, stage times printed)."""
    vp = load_package()
    from vortexpasta_b200 import _lib, tuning
    L = 2 * math.pi
    cases = []
    if args.kernel_case == "pairs1m":
        fs = vp.configs.tangle(5000, 200, 42)
        cases = [("fp64", vp.configs.params_for(L / 16, 4.0, 64, 5)),
                 ("mixed", vp.configs.params_for(L / 16, 4.0, 64, 5, precision="mixed"))]
    elif args.kernel_case == "tuned1m":
        from vortexpasta_b200 import learned
        from vortexpasta_b200.params import C_RTOL_KB
        fs = vp.configs.tangle(5000, 200, 42)
        beta = -math.log(1e-5 / learned.KB_MARGIN / C_RTOL_KB)
        ch = tuning.kb_choice_from(L, 0.139555577934889, beta, 1.5, 3)
        cases = [("mixed", ch.params(L, "mixed"))]
    else:
        fs = vp.configs.tangle(2500, 200, 42)
        ch = tuning.EwaldChoice(alpha=22.0286100737363, rcut=0.15608485585182466, Ns=341, sigma=1.5, m=3)
        cases = [("mixed", ch.params(L, "mixed"))]
    for name, p in cases:
        c = vp.init_cache(p)
        try:
            if args.pair_block:
                _lib.check(_lib.load().vpbs_pair_block(c.handle, args.pair_block), c.handle, "pair_block")
            c.set_filaments(fs)
            c.stage_timing(True)
            for _ in range(3):
                c.compute(_lib.VELOCITY)
                st = c.stage_times()
            print(json.dumps({"case": args.kernel_case, "form": name, "stages_ms": st,
                              "pairs": list(c.pair_counts())}), flush=True)
        finally:
            c.close()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="tangle1m", choices=sorted(WORKLOAD_DESC))
    ap.add_argument("--cpu-reps", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-mixed", dest="mixed", action="store_false",
                    help="skip the mixed-precision (FP32 bulk) form reported under 'forms'")
    ap.add_argument("--no-tuned", dest="tuned", action="store_false",
                    help="skip the tuned form (learned parameters); the headline is then the plain FP64 form")
    ap.add_argument("--rtol", type=float, default=1e-5, help="accuracy target of the tuned form")
    ap.add_argument("--ensemble-steps", type=int, default=20,
                    help="RK4 steps of the batching-form ensemble reported under 'ensemble' (0: skip)")
    ap.add_argument("--kernel-case", choices=sorted(KERNEL_CASES), default=None,
                    help="run a small fixed workload for kernel profiling instead of the benchmark")
    ap.add_argument("--pair-block", type=int, default=0,
                    help="with --kernel-case: the pair kernel's cells per CTA edge (0: the built-in rule)")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "ours":
        print("warning: fewer than 3 warm-up steps", file=sys.stderr)
    if args.kernel_case:
        return run_kernel_case(args)
    rc = check_world(args.gpus)
    if rc is not None:
        return rc
    return run_reference(args) if args.impl == "reference" else run_ours(args)


def launch_command(gpus: int, argv, port: int) -> list:
    """The torchrun command that runs this script with one rank per GPU (loopback rendezvous)."""
    return [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={gpus}",
            "--master-addr=127.0.0.1", f"--master-port={port}", str(Path(__file__).resolve()), *argv]


def check_world(gpus: int):
    """--gpus N: under torchrun the world size must be N (else an error); without torchrun and N > 1
    the script relaunches itself with one rank per GPU and returns that run's exit code.  None: run
    here."""
    if gpus < 1:
        print("bench.py: --gpus must be >= 1", file=sys.stderr)
        return 2
    world_env = os.environ.get("WORLD_SIZE")
    if world_env is not None:
        if int(world_env) != gpus:
            print(f"bench.py: --gpus {gpus} but the launcher started {world_env} ranks", file=sys.stderr)
            return 2
        return None
    if gpus == 1:
        return None
    import socket
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    return subprocess.call(launch_command(gpus, sys.argv[1:], port))


if __name__ == "__main__":
    sys.exit(main())
