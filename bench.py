"""Benchmark of the split-solver step on B200: cell-updates/s and % of the HBM
roofline.

Workload (one bench step): the 2-D four-quadrant Riemann problem on a
4096 x 4096 grid over [0,1]^2, gamma = 1.4, quadrant states (rho, u, v, p)
drawn from the seed (rho log-uniform in [0.1, 10], velocities uniform in
[-2, 2], p log-uniform in [0.01, 1000]); dimensionally split MUSCL-Hancock
with the van Leer limiter and pressure flattening, HLLC flux, FP64,
transmissive boundaries, 100 time steps at CFL 0.8, the CFL reduction fused
into the last sweep of each step.  Synthetic data (seeded), inputs resident
in HBM when timing starts; each 537 MB state buffer exceeds the 126 MB L2.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Under torchrun (N > 1) the ranks solve one grid of size x (size * N) cells,
split into N slabs of rows (each GPU keeps a size^2 slab: weak scaling); 4
ghost rows are exchanged with the neighbouring ranks over NCCL before every
sweep and the CFL maximum is MAX-reduced once per step.  The line reports the
aggregate over ranks, timed as the max over ranks.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

GAMMA = 1.4
SEED = 0
# DRAM bytes (read + write) per cell of one sweep launch, measured by ncu at
# 4096^2 on four consecutive launches of the headline loop (FP64 HLLC,
# staged_walk_2d x and y sweeps of the alternating-layout loop: 608.6 MB read
# + 496.1 MB written per launch on average, 1,104.7 MB against 1,073.7 MB
# algorithmic; profiles/staged_walk_2d_f64_hllc_4096sq.md).
MEASURED_TRAFFIC_PER_CELL = {("f64", "hllc"): 1104.7e6 / 4096 ** 2}


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--size", type=int, default=4096)
    p.add_argument("--time-steps", type=int, default=100)
    p.add_argument("--dtype", choices=["f64", "f32"], default="f64")
    p.add_argument("--flux", choices=["hllc", "force"], default="hllc")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-variants", action="store_true")
    p.add_argument("--no-batched", action="store_true")
    p.add_argument("--no-adjoint", action="store_true")
    p.add_argument("--no-mm", action="store_true")
    p.add_argument("--no-e2e", action="store_true",
                   help="skip the end-to-end host-buffer leg (profiling captures)")
    p.add_argument("--no-correctness", action="store_true",
                   help="skip the L1-vs-FP64 and conservation figures")
    p.add_argument("--mm-steps", type=int, default=500)
    p.add_argument("--slab-impl", choices=["native", "python"], default="native",
                   help="N > 1: the decomposed step through fl_slab_steps (NCCL, one call per "
                        "run) or the Python schedule over fl_sim_sweep and torch.distributed")
    p.add_argument("--only", choices=["mm", "adjoint", "batched", "3d"], default=None,
                   help="run one secondary workload alone (profiling); prints its own line")
    p.add_argument("--size-3d", type=int, default=256, help="--only 3d: cells per side")
    p.add_argument("--steps-3d", type=int, default=20, help="--only 3d: time steps per run")
    return p.parse_args()


def workload_config(a):
    return {
        "workload": f"2-D four-quadrant Riemann problem {a.size}x{a.size} on [0,1]^2, "
                    f"{a.time_steps} steps, MUSCL-Hancock + van Leer + flattening, "
                    f"{a.flux.upper()} flux, CFL 0.8, transmissive",
        "grid": [a.size, a.size],
        "time_steps_per_run": a.time_steps,
        "flux": a.flux,
        "limiter": "vanleer",
        "reconstruction": "muscl-hancock",
        "seed": SEED,
        "l2": "no flush: every state buffer (%d MB) exceeds the 126 MB L2"
              % (a.size * a.size * 4 * (8 if a.dtype == "f64" else 4) // 2 ** 20),
        "parallelism": "replicas" if a.gpus > 1 else "single",
    }


def alternating_transposes(a):
    """Plane transposes per run of the device-resident loop: the 2-D loop in
    FP64, and in FP32 with HLLC, alternates layouts (state in, then back out)
    when both extents are multiples of 16 bytes and no FLUIDITY_B200_SWEEP
    override is set; "staged" extends it to every dtype and flux."""
    mode = os.environ.get("FLUIDITY_B200_SWEEP", "")
    elem = 8 if a.dtype == "f64" else 4
    on = (mode == "staged") or (mode == "" and (a.dtype == "f64" or a.flux == "hllc"))
    return 2 if on and (a.size * elem) % 16 == 0 else 0


def sweep_kernel_name(a):
    if alternating_transposes(a):
        return ("staged_walk_2d (x and y sweeps, averaged; each sweep reads its input with "
                "its own dimension slowest and writes it transposed)")
    return "walk_kernel_2d (x and y sweeps, averaged)"


# ---- distributed plumbing ---------------------------------------------------

def dist_init(a):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        backend = "nccl" if a.impl == "ours" else "gloo"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, world, device=None):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ---- clocks ---------------------------------------------------------------

class ClockSampler:
    """nvidia-smi samples during the timed region."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.lines = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100", "-i", str(self.gpu)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, ValueError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, power, reasons = [], [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
                power.append(float(f[3]))
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax),
                "power_w_max": max(power), "samples": len(sm), "reasons": sorted(reasons)}


# ---- CPU baseline (reference functors) -------------------------------------

def cpu_reference_rate(a, budget_s=12.0, max_steps=50):
    """Times the reference's own numerics functors on the host cores on a
    bounded sample of the workload: whole time steps of the same grid, starting
    from the same initial state.  Returns (cell-updates/s, kind, cores, sample)."""
    from oracle import oracle
    from fluidity_b200.workloads import riemann_states
    shape = (a.size, a.size)
    u = oracle.fill_riemann(shape, riemann_states(SEED, 2), GAMMA)
    cells = a.size * a.size
    cores = os.cpu_count() or 1
    if oracle.ref_available():
        kind = "reference"
        run = lambda n: oracle.ref_simulate(shape, u, GAMMA, 0.8, 1.0 / a.size, 1e30, n,
                                            flux=a.flux)
    else:
        kind = "port"
        cores = 1
        run = lambda n: oracle.simulate(shape, u, GAMMA, 0.8, 1.0 / a.size, 1e30, n,
                                        flux=a.flux)
    t0 = time.perf_counter()
    run(1)
    t1 = time.perf_counter() - t0
    n = int(max(1, min(max_steps, budget_s / max(t1, 1e-6))))
    t0 = time.perf_counter()
    run(n)
    dt = time.perf_counter() - t0
    sample = (f"{n} time step(s) of the {a.size}x{a.size} FP64 {a.flux.upper()} run from its "
              f"initial state, {cores} thread(s), {dt:.1f} s")
    return cells * n / dt, kind, cores, sample


def run_reference_arm(a, world, rank):
    if rank != 0:
        return
    if a.dtype != "f64":
        print(json.dumps({"impl": "reference", "unavailable":
                          "the reference's MUSCL reconstructor does not compile for float"}))
        return
    from oracle import oracle
    from fluidity_b200.workloads import riemann_states
    shape = (a.size, a.size)
    cells = a.size * a.size
    u = oracle.fill_riemann(shape, riemann_states(SEED, 2), GAMMA)
    if oracle.ref_available():
        kind, cores = "reference", os.cpu_count() or 1
        step = lambda: oracle.ref_simulate(shape, u, GAMMA, 0.8, 1.0 / a.size, 1e30, 1,
                                           flux=a.flux)
    else:
        kind, cores = "port", 1
        step = lambda: oracle.simulate(shape, u, GAMMA, 0.8, 1.0 / a.size, 1e30, 1, flux=a.flux)
    for _ in range(a.warmup):
        step()
    t0 = time.perf_counter()
    for _ in range(a.steps):
        step()
    dt = time.perf_counter() - t0
    value = cells * a.steps / dt
    sample = (f"each step: one time step (both sweeps + CFL) of the {a.size}x{a.size} FP64 "
              f"{a.flux.upper()} run, {cores} thread(s)")
    line = {
        "impl": "reference", "metric": "cell-updates/s", "value": value,
        "unit": "cell-updates/s", "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": dt / a.steps * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": a.dtype, "data": "synthetic",
        "config": workload_config(a),
        "cpu_baseline": {"value": value, "unit": "cell-updates/s", "cores": cores,
                         "kind": kind, "sample": sample},
        "e2e": {"value": value, "unit": "cell-updates/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


# ---- our arm ------------------------------------------------------------------

def run_ours(a, world, rank, local):
    import torch
    from fluidity_b200 import build as fb
    fb.build()
    from fluidity_b200.solver import Simulation, SplitSolver
    from fluidity_b200.workloads import riemann_states

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    shape = (a.size, a.size)
    cells = a.size * a.size
    T = a.time_steps
    states = riemann_states(SEED, 2)
    s = SplitSolver(shape, dtype=a.dtype, flux=a.flux, limiter="vanleer", gamma=GAMMA)
    buf_a = s.new_state()
    buf_b = s.new_state()
    sim = Simulation(s)
    stream = torch.cuda.current_stream()

    def one_run(events=None):
        s.fill_riemann(states, out=buf_a)
        sim.begin(buf_a, buf_b, 0.8, 1.0 / a.size, 1e30, T)
        if events is not None:
            events[0].record(stream)
        sim.steps(T)
        if events is not None:
            events[1].record(stream)

    for _ in range(a.warmup):
        one_run()
    it, _, done, _ = sim.status()
    if it != T:
        raise RuntimeError(f"warm-up run stopped after {it} of {T} steps (non-finite state?)")

    sampler = ClockSampler(local)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(a.steps)]
    barrier(world)
    torch.cuda.synchronize()
    sampler.start()
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    t_start.record(stream)
    for k in range(a.steps):
        one_run(ev[k])
    t_end.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    clocks = sampler.stop()
    elapsed_ms = t_start.elapsed_time(t_end)
    sweep_ms = sum(e0.elapsed_time(e1) for e0, e1 in ev)
    it, _, done, _ = sim.status()
    if it != T:
        raise RuntimeError(f"timed run stopped after {it} of {T} steps")
    elapsed_ms = max_over_ranks(elapsed_ms, world, dev)

    elem = 8 if a.dtype == "f64" else 4
    nc = 4
    launches_per_run = 2 * T
    sweep_s = sweep_ms / 1e3 / (a.steps * launches_per_run)
    bytes_per_sweep = 2 * nc * elem * cells          # one read + one write of the state
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(peaks_path):
        peak = json.load(open(peaks_path))["hbm_gbs"]
        peak_src = "measured"
    else:
        peak, peak_src = 6650.0, "fallback"
    achieved = bytes_per_sweep / sweep_s / 1e9
    value = world * cells * T * a.steps / (elapsed_ms / 1e3)

    # ---- end to end through the C ABI with host buffers ----------------------
    # fl_host_pipe_run: each step is one whole simulation from a pinned host
    # state to a pinned host result; job k + 1's upload and job k - 1's
    # download overlap job k's compute.  Every step's copies are inside the
    # timed region; the first upload and the last download are not hidden.
    from fluidity_b200.solver import HostPipeline
    state_bytes = nc * elem * cells
    e2e_steps, e2e_value = 0, None
    if not a.no_e2e:
        pinned_in = torch.empty(buf_a.shape, dtype=buf_a.dtype, pin_memory=True)
        s.fill_riemann(states, out=buf_a)
        pinned_in.copy_(buf_a)
        torch.cuda.synchronize()
        # the same K steps as the device-timed leg; results land in three
        # pinned buffers in turn (a buffer's download k finishes before
        # download k + 3 starts: downloads run in order on one stream)
        e2e_steps = max(2, a.steps)
        pinned_out = [torch.empty(buf_a.shape, dtype=buf_a.dtype, pin_memory=True)
                      for _ in range(min(e2e_steps, 3))]
        pipe = HostPipeline(s, sets=3)
        pipe.run([pinned_in], pinned_out[:1], 0.8, 1.0 / a.size, 1e30, T)     # warm-up
        barrier(world)
        t0 = time.perf_counter()
        jobs = pipe.run([pinned_in] * e2e_steps,
                        [pinned_out[k % len(pinned_out)] for k in range(e2e_steps)],
                        0.8, 1.0 / a.size, 1e30, T)
        e2e_s = time.perf_counter() - t0
        e2e_s = max_over_ranks(e2e_s, world, dev)
        if any(it2 != T for it2, _ in jobs):
            raise RuntimeError("end-to-end run did not complete")
        e2e_value = world * cells * T * e2e_steps / e2e_s
        del pipe

    drop_in = measure_drop_in(a, s, states, sweep_s)
    variants = {}
    ref_cache = {}
    headline_checks = None
    if rank == 0 and world == 1 and not a.no_correctness:
        headline_checks = correctness(2, a.size, a.dtype, a.flux, ref_cache)
    if not a.no_variants and rank == 0:
        for dt_, fx in (("f64", "hllc"), ("f32", "hllc"), ("f64", "force"), ("f32", "force")):
            if (dt_, fx) == (a.dtype, a.flux):
                continue
            variants[f"{fx}_{dt_}"] = measure_variant(a, dt_, fx, states)
            if not a.no_correctness:
                variants[f"{fx}_{dt_}"].update(correctness(2, a.size, dt_, fx, ref_cache))
        for fx in ("hllc", "force"):
            for dt_ in ("f64", "f32"):
                variants[f"3d_{fx}_{dt_}"] = measure_3d(dt_, flux=fx)
                if not a.no_correctness:
                    variants[f"3d_{fx}_{dt_}"].update(correctness(3, 256, dt_, fx, ref_cache))

    line = {
        "metric": "cell-updates/s", "value": value, "unit": "cell-updates/s",
        "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": elapsed_ms / a.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": a.dtype, "data": "synthetic",
        "config": workload_config(a),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak,
                     "traffic": (MEASURED_TRAFFIC_PER_CELL[(a.dtype, a.flux)] * cells
                                 if (a.dtype, a.flux) in MEASURED_TRAFFIC_PER_CELL else None),
                     "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum, "
                                       "average over 4 sweep launches of the 4096^2 loop, "
                                       "per cell (scaled to this grid when it differs)",
                     "kernel": sweep_kernel_name(a),
                     "algorithmic_bytes_per_launch": bytes_per_sweep,
                     "launch_ms": sweep_s * 1e3, "peak_source": peak_src},
        "e2e": {"value": e2e_value, "unit": "cell-updates/s",
                "h2d_bytes_per_step": state_bytes, "d2h_bytes_per_step": state_bytes,
                "steps": e2e_steps, "api": "fl_host_pipe_run (pinned host in/out)",
                "overlap": "upload of step k+1 and download of step k-1 run during step k"},
        "gpu_launches": a.steps * (3 + launches_per_run + alternating_transposes(a)),
        "clocks": clocks,
    }
    line["drop_in"] = drop_in
    if headline_checks is not None:
        line.update(headline_checks)
    if variants:
        line["variants"] = variants
    if rank == 0 and world == 1 and not a.no_batched:
        line["batched"] = measure_batched()
    if rank == 0 and world == 1 and not a.no_adjoint:
        line["adjoint"] = measure_adjoint()
    if rank == 0 and world == 1 and not a.no_mm:
        line["multimaterial"] = measure_multimaterial(steps=a.mm_steps,
                                                      cpu=not a.no_cpu_baseline)
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        v, kind, cores, sample = cpu_reference_rate(a)
        line["cpu_baseline"] = {"value": v, "unit": "cell-updates/s", "cores": cores,
                                "kind": kind, "sample": sample}
    if rank == 0:
        print(json.dumps(line))
    del sim


def measure_drop_in(a, s, states, loop_sweep_s, steps=20):
    """The drop-in step on the headline grid: fl_split_solve_ws (the
    reference's SplitSolver::solve interface with a caller-owned workspace)
    for `steps` steps at the initial CFL time step, timed with CUDA events;
    per-sweep time against the device-resident loop's."""
    import torch
    x, y = s.new_state(), s.new_state()
    s.fill_riemann(states, out=x)
    dtdh = 0.8 / s.max_wavespeed(x).item()
    mws = torch.zeros(1, dtype=torch.float64, device="cuda")
    for _ in range(2):                                   # warm-up
        x, y = s.solve(x, y, dtdh, max_ws=mws)[::-1]
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        x, y = s.solve(x, y, dtdh, max_ws=mws)[::-1]
    e1.record()
    torch.cuda.synchronize()
    sweep_ms = e0.elapsed_time(e1) / (steps * len(s.shape))
    del x, y
    torch.cuda.empty_cache()
    return {"api": "fl_split_solve_ws (caller-owned workspace, strips taken dynamically)",
            "steps": steps, "sweep_ms": sweep_ms, "loop_sweep_ms": loop_sweep_s * 1e3,
            "ratio_to_loop": sweep_ms / (loop_sweep_s * 1e3)}


def measure_variant(a, dtype, flux, states, runs=3):
    import torch
    from fluidity_b200.solver import Simulation, SplitSolver
    s = SplitSolver((a.size, a.size), dtype=dtype, flux=flux, gamma=GAMMA)
    x = s.new_state()
    y = s.new_state()
    sim = Simulation(s)
    T = a.time_steps
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    total = 0.0
    for k in range(runs + 1):
        s.fill_riemann(states, out=x)
        sim.begin(x, y, 0.8, 1.0 / a.size, 1e30, T)
        e0.record()
        sim.steps(T)
        e1.record()
        torch.cuda.synchronize()
        if k > 0:
            total += e0.elapsed_time(e1)
    it, _, _, _ = sim.status()
    elem = 8 if dtype == "f64" else 4
    sweep_s = total / 1e3 / (runs * 2 * T)
    cells = a.size * a.size
    return {"cell_updates_per_s": cells * T * runs / (total / 1e3),
            "sweep_gbs": 2 * 4 * elem * cells / sweep_s / 1e9, "steps_completed": it}


def measure_3d(dtype, flux="hllc", n=256, steps=20, runs=3):
    """3-D octant Riemann problem n^3 (the config's 3-D variant): steps HLLC /
    van Leer MUSCL-Hancock steps at CFL 0.8 through the tile kernel, 3 sweeps a
    step.  Reports cell-updates/s and each sweep's algorithmic bytes (one read
    and one write of the 5-component state) against the measured HBM peak."""
    import torch
    from fluidity_b200.solver import Simulation, SplitSolver
    from fluidity_b200.workloads import riemann_states
    s = SplitSolver((n, n, n), dtype=dtype, flux=flux, gamma=GAMMA)
    x = s.new_state()
    y = s.new_state()
    sim = Simulation(s)
    st = riemann_states(SEED, 3)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    total = 0.0
    for k in range(runs + 1):
        s.fill_riemann(st, out=x)
        sim.begin(x, y, 0.8, 1.0 / n, 1e30, steps)
        e0.record()
        sim.steps(steps)
        e1.record()
        torch.cuda.synchronize()
        if k > 0:
            total += e0.elapsed_time(e1)
    it, _, _, _ = sim.status()
    elem = 8 if dtype == "f64" else 4
    cells = n ** 3
    sweep_s = total / 1e3 / (runs * 3 * steps)
    gbs = 2 * 5 * elem * cells / sweep_s / 1e9
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    peak = json.load(open(peaks_path))["hbm_gbs"] if os.path.exists(peaks_path) else 6650.0
    return {"workload": f"3-D octant Riemann problem {n}^3, {steps} steps, {flux.upper()}",
            "cell_updates_per_s": cells * steps * runs / (total / 1e3), "sweep_gbs": gbs,
            "frac_of_measured_hbm": gbs / peak, "steps_completed": it}


PARITY_BARS = {
    "f64": "1e-12 relative per cell and sweep against the reference's functors "
           "(relative to max(|ref|, 1e-3 of the component's largest magnitude))",
    "f32": "1e-5 of the component's largest magnitude per cell and sweep against the FP32 "
           "restatement of the reference's arithmetic",
}


def correctness(dims, n, dtype, flux, ref_cache, steps=2):
    """Per-result correctness figures of one workload variant.

    l1_vs_fp64: relative L1 per component (sum |x - ref| / sum |ref|) of the
    state after `steps` time steps of the run (device-resident loop, same
    kernels as the timed run) against the FP64 reference run of the same
    steps from the same initial data: the reference's own functors
    (oracle/_ref) on the host cores, or the pinned C oracle where that
    library is absent.

    conservation: for each sweep of those steps, the residual of
    sum U_out - sum U_in - dtdh (inflow - outflow) per component, relative to
    sum |U_in| + the boundary flux magnitudes (fluidity_b200/diagnostics.py):
    mass, momentum and energy change only by the flux through the
    transmissive ends, to round-off."""
    import torch
    from oracle import oracle
    from fluidity_b200.diagnostics import l1_relative, sweep_conservation_residual
    from fluidity_b200.solver import Simulation, SplitSolver
    from fluidity_b200.workloads import riemann_states
    shape = (n,) * dims
    st = riemann_states(SEED, dims)
    key = (dims, n, flux, steps)
    if key not in ref_cache:
        u0 = oracle.fill_riemann(shape, st, GAMMA)
        t0 = time.perf_counter()
        if oracle.ref_available():
            ref, k, _, _ = oracle.ref_simulate(shape, u0, GAMMA, 0.8, 1.0 / n, 1e30, steps,
                                               flux=flux)
            kind = "reference functors (oracle/_ref)"
        else:
            ref, k, _, _ = oracle.simulate(shape, u0, GAMMA, 0.8, 1.0 / n, 1e30, steps, flux=flux)
            kind = "C oracle (pinned to the reference's functors)"
        ref_cache[key] = (torch.from_numpy(ref), k, kind, time.perf_counter() - t0)
        del u0
    ref, k, kind, ref_s = ref_cache[key]
    s = SplitSolver(shape, dtype=dtype, flux=flux, gamma=GAMMA)
    a = s.fill_riemann(st)
    b = torch.empty_like(a)
    res, it, _ = Simulation(s).run(a, b, 0.8, 1.0 / n, 1e30, steps)
    l1 = l1_relative(res.cpu(), ref, shape)
    # conservation of each sweep of the same steps
    a = s.fill_riemann(st)
    worst = {}
    for _ in range(steps):
        dtdh = 0.8 / s.max_wavespeed(a).item()
        for dim in range(dims):
            s.sweep(a, b, dim, dtdh)
            for c, v in sweep_conservation_residual(shape, a, b, dim, dtdh, GAMMA).items():
                worst[c] = max(worst.get(c, 0.0), v)
            a, b = b, a
    torch.cuda.synchronize()
    del a, b, res, s
    torch.cuda.empty_cache()
    return {
        "l1_vs_fp64": {"steps": int(it), "reference": kind, "reference_steps": int(k),
                       "per_component": {c: float(f"{v:.3g}") for c, v in l1.items()}},
        "conservation": {"sweeps": steps * dims, "max_rel_residual":
                         {c: float(f"{v:.3g}") for c, v in worst.items()},
                         "check": "sum U_out - sum U_in - dtdh * (flux through the "
                                  "transmissive ends) per sweep, over sum |U_in|"},
        "parity_bar": PARITY_BARS[dtype],
    }


def measure_batched(seed=3, steps=200, baseline_every=4):
    """Batched workload: 3584 1-D problems (cells log-uniform in [64, 8192]) and
    512 2-D problems (side log-uniform in [64, 512]), FP32 HLLC + van Leer, CFL
    0.8, 200 steps each.  The batched solver (autotuned, time loop captured in
    one CUDA graph) against per-problem launches of the plain step (fl_sim_*
    per problem, all on one stream), the latter timed on every
    `baseline_every`-th problem and reported as a rate."""
    import torch
    from fluidity_b200.batch import Batch, batched_workload
    from fluidity_b200.solver import Simulation, SplitSolver
    probs = batched_workload(seed=seed)
    b = Batch(probs, dtype="f32", flux="hllc")
    b.fill()
    t0 = time.perf_counter()
    tune = b.autotune(trial_steps=8)
    tune_s = time.perf_counter() - t0
    b.fill()
    b.begin(0.8, 1e30, steps)
    b.capture(steps)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    runs = []
    for k in range(3):                     # first replay is the warm-up
        b.fill()
        torch.cuda.synchronize()
        e0.record()
        b.begin(0.8, 1e30, steps)
        b.launch()
        e1.record()
        torch.cuda.synchronize()
        runs.append(e0.elapsed_time(e1))
    it, _, done, rc = b.status(allow_nan=True)
    ms = min(runs[1:])
    cells = np.array([int(np.prod(s)) for s, _ in probs])
    updates = float(np.sum(cells * it))
    rate = updates / (ms / 1e3)
    # per-problem launches of the plain step
    sub = list(range(0, len(probs), baseline_every))
    b.fill()
    sims = []
    for i in sub:
        shape = probs[i][0]
        s = SplitSolver(shape, dtype="f32", flux="hllc", pitch=b.pitches[i])
        sims.append((s, Simulation(s), b.state(i, b.a), b.state(i, b.b)))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for s, sim, x, y in sims:
        sim.begin(x, y, 0.8, 1.0 / s.shape[0], 1e30, steps)
        sim.steps(steps)
    torch.cuda.synchronize()
    base_s = time.perf_counter() - t0
    base_updates = 0.0
    for (s, sim, x, y) in sims:
        itb, _, _, _ = sim.status(allow_nan=True)
        base_updates += float(np.prod(s.shape)) * itb
    base_rate = base_updates / base_s
    return {
        "workload": "4096 problems: 3584 1-D (n log-uniform [64, 8192]) + 512 2-D "
                    "(side log-uniform [64, 512]), FP32 HLLC + van Leer, CFL 0.8, 200 steps",
        "cell_updates_per_s": rate, "ms_per_run": ms, "cell_updates": updates,
        "problems_finished": int(done), "problems_stopped_nonfinite": int(np.sum(it < steps)),
        "per_problem_launch_cell_updates_per_s": base_rate,
        "per_problem_sample": f"every {baseline_every}th problem ({len(sub)} problems), "
                              f"{base_s:.2f} s",
        "speedup_vs_per_problem": rate / base_rate,
        "autotune": tune, "autotune_s": tune_s, "graph": True,
    }


def _fd_check(adj, rho0, grad, p_target, directions, eps, seed=7):
    """Relative mismatch, per seeded unit direction, of central differences
    (time steps frozen from the unperturbed forward pass; the difference of J
    formed cell by cell, free of cancellation) against the adjoint's
    directional derivative; NaN where a value is not finite."""
    import torch
    from fluidity_b200.adjoint import objective_difference, random_directions, state_from_density
    dts = adj.dtdh()
    out = []
    with torch.no_grad():
        for v in random_directions(rho0.numel(), directions, seed=seed, dtype=rho0.dtype):
            up = adj.forward(state_from_density(rho0 + eps * v), 0.7, frozen_dtdh=dts)
            um = adj.forward(state_from_density(rho0 - eps * v), 0.7, frozen_dtdh=dts)
            fd = objective_difference(up.double(), um.double(), p_target.double()).item() / (2 * eps)
            ad = torch.dot(grad, v).item()
            r = abs(fd - ad) / max(abs(ad), 1e-300)
            out.append(r if math.isfinite(r) else float("nan"))
    return out


def _fd_summary(errs):
    finite = [e for e in errs if math.isfinite(e)]
    return {"max": max(finite) if len(finite) == len(errs) else float("nan"),
            "median": statistics.median(finite) if finite else float("nan"),
            "below_1e-6": sum(1 for e in finite if e < 1e-6),
            "per_direction": [float(f"{e:.3g}") for e in errs]}


def measure_adjoint(n=1024, steps=300, directions=16, eps=1e-6):
    """Gradient workload: 2-D n x n, density 1 + 32 seeded Gaussians at rest
    with p = rho (temperature 1; with a uniform p the field is an exact steady
    state and the objective would not depend on the density); 300 HLLC/MUSCL
    steps at CFL 0.7; J = 0.5 ||p(T) - p_target||^2 with p_target from a
    second seed's field; dJ/d rho0 by the discrete adjoint with
    ceil(sqrt(300)) = 18-step checkpoints, checked against central differences
    along 16 seeded unit directions (time steps frozen) at eps 1e-6 and 1e-7.
    The discrete step is piecewise smooth (minmod switches, the HLLC
    shock/rarefaction estimate): a direction whose central difference
    straddles a switch mixes two one-sided derivatives, so the check reports
    every direction, not only the worst."""
    import torch
    from fluidity_b200.adjoint import (Adjoint, gaussian_density, objective, pressure, rollout,
                                       state_from_density)
    out = {}
    grads = {}
    for dtype in ("f64", "f32"):
        tdt = torch.float64 if dtype == "f64" else torch.float32
        adj = Adjoint((n, n), steps, dtype=dtype)
        with torch.no_grad():
            p_target = pressure(adj.forward(state_from_density(
                gaussian_density(n, 2, dtype=tdt)), 0.7))
        rho0 = gaussian_density(n, 1, dtype=tdt).requires_grad_(True)
        e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        uN = rollout(state_from_density(rho0), adj, 0.7)   # warm-up (kernel set-up)
        objective(uN, p_target).backward()
        fwd, bwd = [], []
        for _ in range(3):                    # median of three timed rollouts
            rho0.grad = None
            u0 = state_from_density(rho0)
            torch.cuda.synchronize()
            e[0].record()
            uN = rollout(u0, adj, 0.7)
            J = objective(uN, p_target)
            e[1].record()
            J.backward()
            e[2].record()
            torch.cuda.synchronize()
            fwd.append(e[0].elapsed_time(e[1]))
            bwd.append(e[1].elapsed_time(e[2]))
        fwd_ms, bwd_ms = statistics.median(fwd), statistics.median(bwd)
        grad = rho0.grad.detach().clone()
        res = {"forward_ms": fwd_ms, "backward_ms": bwd_ms,
               "forward_ms_runs": fwd, "backward_ms_runs": bwd,
               "cost_ratio_backward_over_forward": bwd_ms / fwd_ms,
               "objective": J.item(), "grad_norm": torch.norm(grad.double()).item()}
        grads[dtype] = grad.double()
        if dtype == "f64":
            e6 = _fd_check(adj, rho0.detach(), grad, p_target, directions, eps)
            e7 = _fd_check(adj, rho0.detach(), grad, p_target, directions, eps / 10)
            res.update({"fd_directions": directions,
                        "fd_eps_1e-6": _fd_summary(e6), "fd_eps_1e-7": _fd_summary(e7),
                        "fd_max_rel_err": max(e6)})
            # the same check without the flattening coefficient, which the
            # adjoint holds frozen: there the adjoint is the exact derivative
            # away from limiter and wave-speed switches
            adj_nf = Adjoint((n, n), steps, dtype=dtype, flatten=False)
            rho_nf = rho0.detach().clone().requires_grad_(True)
            with torch.no_grad():
                pt_nf = pressure(adj_nf.forward(state_from_density(
                    gaussian_density(n, 2, dtype=tdt)), 0.7))
            objective(rollout(state_from_density(rho_nf), adj_nf, 0.7), pt_nf).backward()
            enf = _fd_check(adj_nf, rho_nf.detach(), rho_nf.grad.detach(), pt_nf, directions,
                            eps)
            res["fd_no_flattening_eps_1e-6"] = _fd_summary(enf)
            del adj_nf
        else:
            g64 = grads["f64"]
            res["rel_diff_vs_f64_gradient"] = (torch.norm(grads["f32"] - g64) /
                                               torch.norm(g64)).item()
        out[dtype] = res
    out["workload"] = (f"2-D {n}x{n}, rho0 = 1 + 32 Gaussians, p = rho0, at rest, {steps} "
                       f"HLLC/MUSCL steps at CFL 0.7, checkpoint every "
                       f"{math.ceil(math.sqrt(steps))} steps")
    out["exactness"] = adjoint_exactness()
    return out


def adjoint_exactness(n=128, steps=40, directions=4, eps=1e-6):
    """The FP64 adjoint against an exact reference gradient at a size the CPU
    evaluates: per seeded direction, <adjoint gradient, v> against the
    directional derivative in forward-mode dual numbers through the oracle's
    sweep (oracle/fl_oracle_dual.cpp; the same frozen branches and time
    steps, the flattening coefficient differentiated through its ramp), the
    central difference against that exact value, and the branch decisions
    that differ between u + eps v and u - eps v (oracle.branch_flips).  Where
    the adjoint matches the exact derivative to rounding, a central
    difference that misses it is off by its own errors: limiter and
    wave-speed switches inside +-eps, and round-off in J(u+) - J(u-)."""
    import numpy as np
    import torch
    from oracle import oracle
    from fluidity_b200.adjoint import (Adjoint, gaussian_density, objective,
                                       objective_difference, pressure, random_directions,
                                       rollout, state_from_density)
    adj = Adjoint((n, n), steps, dtype="f64")
    with torch.no_grad():
        p_target = pressure(adj.forward(state_from_density(gaussian_density(n, 2)), 0.7))
    rho0 = gaussian_density(n, 1).requires_grad_(True)
    objective(rollout(state_from_density(rho0), adj, 0.7), p_target).backward()
    grad = rho0.grad.detach()
    dts = adj.dtdh()
    r0 = rho0.detach().cpu().numpy()
    pt = p_target.cpu().numpy()
    z = np.zeros_like(r0)
    u0 = np.stack([r0, r0 / 0.4, z, z])
    t0 = time.perf_counter()
    ad_err, fd_chi_err, chi_terms, flips = [], [], [], []

    def directional(u, du):
        rho, e, mx, my = u
        drho, de, dmx, dmy = du
        ke = 0.5 * (mx * mx + my * my) / rho
        dke = (mx * dmx + my * dmy) / rho - ke * drho / rho
        return float(np.sum((0.4 * (e - ke) - pt) * 0.4 * (de - dke)))

    with torch.no_grad():
        for v in random_directions(r0.size, directions, seed=7):
            vn = v.cpu().numpy()
            dv = np.stack([vn, vn / 0.4, z, z])
            exact = directional(*oracle.rollout_dual((n, n), u0, dv, 1.4, dts))
            exact_chi = directional(*oracle.rollout_dual((n, n), u0, dv, 1.4, dts,
                                                         chi_diff=True))
            _, tp = oracle.rollout_trace((n, n), u0 + eps * dv, 1.4, dts)
            _, tm = oracle.rollout_trace((n, n), u0 - eps * dv, 1.4, dts)
            ad = torch.dot(grad, v).item()
            up = adj.forward(state_from_density(rho0.detach() + eps * v), 0.7, frozen_dtdh=dts)
            um = adj.forward(state_from_density(rho0.detach() - eps * v), 0.7, frozen_dtdh=dts)
            fd = objective_difference(up, um, p_target).item() / (2 * eps)
            ad_err.append(abs(ad - exact_chi) / abs(exact_chi))
            fd_chi_err.append(abs(fd - exact_chi) / abs(exact_chi))
            chi_terms.append(abs(exact_chi - exact) / abs(exact_chi))
            flips.append(oracle.branch_flips(tp, tm))
    del adj
    g3 = lambda xs: [float(f"{e:.3g}") for e in xs]
    return {"grid": f"{n}x{n}", "steps": steps, "reference": "oracle sweep in forward-mode "
            "dual numbers (the forward pass's branches and dt, chi differentiated through its "
            "ramp)", "cpu_s": time.perf_counter() - t0,
            "adjoint_vs_exact_rel": g3(ad_err),
            "central_difference_vs_exact_rel": g3(fd_chi_err),
            "branch_flips_between_u_plus_and_u_minus": flips,
            "chi_terms_rel": g3(chi_terms),
            "reading": "the adjoint equals the exact derivative to rounding; a central "
                       "difference straddling no branch flip equals it too "
                       "(tests/test_branch_flips.py), so the central differences' misses "
                       "here come with flips; chi_terms_rel is the part of the derivative "
                       "that chi's ramp contributes",
            "fd_eps": eps}


def measure_multimaterial(nx=2048, ny=1024, steps=500, reinit_every=5, cpu=True):
    """Two-material shock-bubble workload: 2048 x 1024 on [0,2] x [0,1]
    (h = 1/1024), ambient gamma 1.4 shocked at x = 0.1, bubble gamma 1.67,
    FP32 states, FP64 level sets, HLLC + van Leer MUSCL-Hancock, CFL 0.6,
    WENO-HJ5/RK3 level-set advection, reinitialisation every 5 steps."""
    import torch
    from fluidity_b200.multimaterial import MultiMaterial
    from fluidity_b200.workloads import shock_bubble
    spec = shock_bubble(SEED + 1, nx=nx, ny=ny, width=2.0)
    warm = MultiMaterial.shock_bubble(spec, dtype="f32")
    warm.begin(0.6, 1e30, 3, reinit_every)
    warm.steps(3)
    warm.status()
    del warm
    mm = MultiMaterial.shock_bubble(spec, dtype="f32")
    torch.cuda.synchronize()
    mm.begin(0.6, 1e30, steps, reinit_every)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    mm.steps(steps)
    e1.record()
    it, rt, done = mm.status()
    ms = e0.elapsed_time(e1)
    st = mm.stats()
    u0, u1 = mm.states()
    p0, _ = mm.current_phi()
    finite = bool(torch.isfinite(u0).all().item() and torch.isfinite(u1).all().item())
    cells = nx * ny
    out = {
        "workload": f"2-D two-material shock-bubble {nx}x{ny} on [0,2]x[0,1], Mach "
                    f"{spec['mach']:.3f}, bubble r {spec['radius']:.3f}, FP32 states, FP64 "
                    f"level sets, HLLC + van Leer, CFL 0.6, reinit every {reinit_every} steps",
        "steps": it, "simulated_time": rt, "ms": ms, "ms_per_step": ms / max(it, 1),
        "cell_updates_per_s": cells * it / (ms * 1e-3),
        "material_cell_updates_per_s": 2 * cells * it / (ms * 1e-3),
        "last_step": st, "states_finite": finite,
        "levelset_finite": bool(torch.isfinite(p0).all().item()),
        "levelset_cells_inside_bubble": int((p0 > 0).sum().item()),
    }
    if cpu:
        import time as _t
        import numpy as np
        from oracle import oracle as O
        g0, g1 = spec["gammas"]
        n = cells
        a0 = O.mm_set_states(np.zeros((4, n), np.float32), -np.ones(n), spec["ambient"], g0)
        a0 = O.mm_set_states(a0, spec["shock_phi"], spec["shocked"], g0)
        a1 = O.mm_set_states(np.zeros((4, n), np.float32), -np.ones(n), spec["bubble"], g1)
        p0h, p1h = spec["phi0"], spec["phi1"]
        # one reinitialisation cycle: reinit_every steps, the last followed
        # by the reinitialisation of level set 0; level set 1 takes its
        # negation (the projection leaves phi1 = -phi0 and the
        # reinitialisation is odd), as the GPU loop does
        with O.threaded():
            cores = O.threads()
            t0 = _t.perf_counter()
            for _ in range(reinit_every):
                a0, a1, p0h, p1h, _dt = O.mm_step(nx, ny, spec["h"], spec["gammas"], 0.6, a0,
                                                  a1, p0h, p1h, reinit=False)
            p0h, sweeps = O.ls_reinit(nx, ny, p0h, spec["h"])
            p1h = -p0h
            sec = _t.perf_counter() - t0
        k = reinit_every
        out["cpu_baseline"] = {"value": cells * k / sec, "unit": "cell-updates/s",
                               "cores": cores, "kind": "port",
                               "sample": f"{k} steps and one reinitialisation ({sweeps} Jacobi "
                                         f"sweeps) of the same workload in the C oracle, OpenMP "
                                         f"over rows, {cores} threads, {sec:.1f} s"}
    return out


def run_slabs(a, world, rank, local):
    """N > 1: one 2-D grid of a.size x (a.size * N) cells split into N slabs
    of rows, one per GPU (weak scaling: each GPU keeps an a.size^2 slab).
    Before the x sweep the ranks exchange 3 ghost rows with their neighbours
    over NCCL, before the y sweep 4; the CFL maximum is MAX-reduced once per
    step.  --slab-impl native (default): the whole step enqueued by
    fl_slab_steps; python: the same schedule driven from Python."""
    import torch
    from fluidity_b200 import build as fb
    fb.build()
    from fluidity_b200 import capi
    from fluidity_b200.slab import CudaSlabOps, NativeSlabs, SlabLayout, SlabRunner
    from fluidity_b200.solver import SplitSolver
    from fluidity_b200.workloads import riemann_states

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    nx, ny = a.size, a.size * world
    T = a.time_steps
    L = SlabLayout((nx, ny), world, rank)
    native = a.slab_impl == "native" and bool(capi.load().fl_slab_nccl_available())
    if native:
        ns = NativeSlabs.nccl(L, dtype=a.dtype, flux=a.flux, gamma=GAMMA)
        buf_a, buf_b = ns.new_state(), ns.new_state()

        class _Run:
            def begin(self, x, y, cfl, res, t_end, n):
                ns.begin([x], [y], cfl, res, t_end, n)

            def steps(self, n):
                ns.steps(n)

        runner = _Run()

        def status():
            it, rt, done = ns.status()
            return it, rt, done, None
    else:
        ops = CudaSlabOps(L, dtype=a.dtype, flux=a.flux, gamma=GAMMA)
        runner = SlabRunner(L, ops)
        buf_a, buf_b = ops.new_state(), ops.new_state()
        status = ops.status
    glob = SplitSolver((nx, ny), dtype=a.dtype, flux=a.flux, limiter="vanleer", gamma=GAMMA)
    init = glob.fill_riemann(riemann_states(SEED, 2))[:, L.global_slice()].contiguous()
    del glob
    torch.cuda.empty_cache()
    stream = torch.cuda.current_stream()
    res = 1.0 / nx

    def one_run(events=None):
        buf_a.copy_(init)
        runner.begin(buf_a, buf_b, 0.8, res, 1e30, T)
        if events is not None:
            events[0].record(stream)
        runner.steps(T)
        if events is not None:
            events[1].record(stream)

    for _ in range(a.warmup):
        one_run()
    it, _, _, _ = status()
    if it != T:
        raise RuntimeError(f"warm-up run stopped after {it} of {T} steps")
    sampler = ClockSampler(local)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(a.steps)]
    barrier(world)
    torch.cuda.synchronize()
    sampler.start()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for k in range(a.steps):
        one_run(ev[k])
    t1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    clocks = sampler.stop()
    elapsed_ms = max_over_ranks(t0.elapsed_time(t1), world, dev)
    loop_ms = max_over_ranks(sum(e0.elapsed_time(e1) for e0, e1 in ev), world, dev)
    it, _, _, _ = status()
    if it != T:
        raise RuntimeError(f"timed run stopped after {it} of {T} steps")
    value = nx * ny * T * a.steps / (elapsed_ms / 1e3)
    elem = 8 if a.dtype == "f64" else 4
    sweep_s = loop_ms / 1e3 / (a.steps * 2 * T)
    bytes_per_sweep = 2 * 4 * elem * L.cells
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    peak, peak_src = ((json.load(open(peaks_path))["hbm_gbs"], "measured")
                      if os.path.exists(peaks_path) else (6650.0, "fallback"))
    achieved = bytes_per_sweep / sweep_s / 1e9

    # end to end: the slab from pinned host memory, the run, the slab back
    pin_in = torch.empty(buf_a.shape, dtype=buf_a.dtype, pin_memory=True)
    pin_out = torch.empty(buf_a.shape, dtype=buf_a.dtype, pin_memory=True)
    pin_in.copy_(init)
    e2e_steps = max(2, min(a.steps, 5))

    def e2e_run():
        buf_a.copy_(pin_in, non_blocking=True)
        runner.begin(buf_a, buf_b, 0.8, res, 1e30, T)
        runner.steps(T)
        pin_out.copy_(buf_a, non_blocking=True)
        torch.cuda.synchronize()

    e2e_run()
    barrier(world)
    ts = time.perf_counter()
    for _ in range(e2e_steps):
        e2e_run()
    e2e_s = max_over_ranks(time.perf_counter() - ts, world, dev)
    state_bytes = int(buf_a.numel()) * elem
    if rank == 0:
        line = {
            "metric": "cell-updates/s", "value": value, "unit": "cell-updates/s",
            "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": elapsed_ms / a.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": a.dtype, "data": "synthetic",
            "config": {**workload_config(a),
                       "workload": f"2-D four-quadrant Riemann problem {nx}x{ny} ({nx}^2 per "
                                   f"GPU), {T} steps, MUSCL-Hancock + van Leer + flattening, "
                                   f"{a.flux.upper()} flux, CFL 0.8, transmissive; {world} "
                                   f"slabs of rows, 3 ghost rows exchanged before the x sweep "
                                   f"and 4 before the y sweep",
                       "grid": [nx, ny], "parallelism": f"slab{world}",
                       "slab_step": "fl_slab_steps (NCCL)" if native
                       else "Python schedule over fl_sim_sweep"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": None,
                         "kernel": "the sweep kernels per rank, time per sweep including the "
                                   "ghost-row exchange and the CFL all-reduce",
                         "algorithmic_bytes_per_launch": bytes_per_sweep,
                         "launch_ms": sweep_s * 1e3, "peak_source": peak_src},
            "e2e": {"value": nx * ny * T * e2e_steps / e2e_s, "unit": "cell-updates/s",
                    "h2d_bytes_per_step": state_bytes * world,
                    "d2h_bytes_per_step": state_bytes * world},
            "gpu_launches": a.steps * (3 * T + 3),
            "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    if native:
        torch.cuda.synchronize()
        ns.close()


def run_section(a, local):
    """One secondary workload on its own (for profiling captures)."""
    import torch
    from fluidity_b200 import build as fb
    fb.build()
    torch.cuda.set_device(local)
    if a.only == "mm":
        res = measure_multimaterial(steps=a.mm_steps, cpu=not a.no_cpu_baseline)
    elif a.only == "adjoint":
        res = measure_adjoint()
    elif a.only == "3d":
        res = {dt: measure_3d(dt, n=a.size_3d, steps=a.steps_3d) for dt in ("f64", "f32")}
    else:
        res = measure_batched()
    print(json.dumps({"section": a.only, **res}), flush=True)


def main():
    a = parse()
    world, rank, local = dist_init(a)
    try:
        if a.impl == "reference":
            run_reference_arm(a, world, rank)
        elif a.only is not None:
            run_section(a, local)
        elif world > 1:
            run_slabs(a, world, rank, local)
        else:
            run_ours(a, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
