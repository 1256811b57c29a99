"""The TMA-staged 2-D sweep (staged_walk_2d, fl_staged.cuh) against the CPU
oracle, and the older 2-D kernels kept behind FLUIDITY_B200_SWEEP.

The staged kernel runs wherever a state's rows and planes are multiples of 16
bytes (x extent a multiple of 2 in FP64, of 4 in FP32); these shapes are
chosen so that it does, in both dtypes: partial warps across the sweep (x or y
extents not multiples of 32), strips shorter than the walk's reach, the
smallest grids the ABI accepts, reflective ends and every policy.  By default
it takes the FP64 y sweep; test_staged_x_sweep_parity_subset reruns this
file's parity cases with FLUIDITY_B200_SWEEP=staged, where it takes both
sweeps in both dtypes.

Bars per sweep as in test_split_gpu.py: FP64 1e-12 relative per cell (floor
1e-3 of the component's magnitude), FP32 1e-5 of the component's magnitude.
"""
import os
import subprocess
import sys

import numpy as np
import pytest

from _util import random_prim, rel_err

pytestmark = pytest.mark.gpu

GAMMA = 1.4
TOL = {"f64": 1e-12, "f32": 1e-5}
FLOOR = {"f64": 1e-3, "f32": 1.0}
NPDT = {"f64": np.float64, "f32": np.float32}
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SHAPES = [(64, 48), (100, 36), (8, 4), (4, 40), (136, 70), (32, 130)]
POLICIES = [
    ("hllc", "vanleer", "muscl", True), ("force", "vanleer", "muscl", True),
    ("lf", "superbee", "muscl", True), ("richtmyer", "vanleer", "muscl", True),
    ("hllc", "superbee", "basic", True), ("hllc", "vanleer", "muscl", False),
]


def _sweeps(shape, dtype, u, dtdh, pol, reflect=0, p_inf=0.0):
    """x then y sweep on the GPU (fl_split_sweep, one strip per warp) and in
    the oracle; returns the worst per-sweep error."""
    import torch
    from fluidity_b200.solver import SplitSolver
    flux, lim, recon, flatten = pol
    s = SplitSolver(shape, dtype=dtype, gamma=GAMMA, flux=flux, limiter=lim, recon=recon,
                    flatten=flatten, boundary_mask=reflect, p_inf=p_inf)
    tdt = torch.float64 if dtype == "f64" else torch.float32
    worst = 0.0
    cur = u
    for dim in (0, 1):
        from oracle import oracle
        if p_inf:
            with oracle.stiffened(p_inf):
                ref = oracle.sweep(shape, dim, cur, NPDT[dtype](GAMMA), NPDT[dtype](dtdh),
                                   flux=flux, limiter=lim, recon=recon, flatten=flatten,
                                   reflect=reflect)
        else:
            ref = oracle.sweep(shape, dim, cur, NPDT[dtype](GAMMA), NPDT[dtype](dtdh), flux=flux,
                               limiter=lim, recon=recon, flatten=flatten, reflect=reflect)
        a = torch.from_numpy(np.ascontiguousarray(cur)).to("cuda", tdt)
        b = torch.empty_like(a)
        s.sweep(a, b, dim, float(NPDT[dtype](dtdh)))
        torch.cuda.synchronize()
        worst = max(worst, rel_err(b.cpu().numpy(), ref, FLOOR[dtype]))
        cur = ref
    return worst


@pytest.mark.parametrize("dtype", ["f64", "f32"])
@pytest.mark.parametrize("shape", SHAPES, ids=lambda s: "x".join(map(str, s)))
@pytest.mark.parametrize("pol", POLICIES, ids=lambda p: "-".join(str(x) for x in p))
def test_staged_policy_sweeps(cuda, oracle, shape, dtype, pol):
    # moderate contrasts: the full value ranges on grids a few cells wide
    # drive the oracle itself to negative pressures
    u = oracle.prim_to_cons(random_prim(shape, 3, smooth=True, mild=True), GAMMA,
                            dtype=NPDT[dtype])
    ws = float(oracle.max_wavespeed(shape, u, NPDT[dtype](GAMMA)))
    assert _sweeps(shape, dtype, u, 0.4 / ws, pol) < TOL[dtype]


@pytest.mark.parametrize("dtype", ["f64", "f32"])
@pytest.mark.parametrize("reflect", [1, 2, 3])
@pytest.mark.parametrize("shape", [(64, 48), (8, 4), (4, 40)], ids=lambda s: "x".join(map(str, s)))
def test_staged_reflective(cuda, oracle, shape, dtype, reflect):
    u = oracle.prim_to_cons(random_prim(shape, 8, smooth=True, mild=True), GAMMA,
                            dtype=NPDT[dtype])
    ws = float(oracle.max_wavespeed(shape, u, NPDT[dtype](GAMMA)))
    assert _sweeps(shape, dtype, u, 0.4 / ws, POLICIES[0], reflect=reflect) < TOL[dtype]


@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_staged_flattening_active(cuda, oracle, dtype):
    """An oblique compressive ramp: chi < 1 in both dimensions, across warp
    boundaries in both sweeps."""
    shape = (64, 48)
    prim = np.zeros((4, 64 * 48))
    x = np.tile(np.arange(64), 48)
    y = np.repeat(np.arange(48), 64)
    w = np.clip((x + y - 50) / 4.0, 0.0, 1.0)
    prim[0] = 3.0 + (0.5 - 3.0) * w
    prim[1] = 20.0 + (1.0 - 20.0) * w
    prim[2] = 1.0 + (-0.5 - 1.0) * w
    prim[3] = 1.0 + (-0.5 - 1.0) * w
    u = oracle.prim_to_cons(prim, GAMMA, dtype=NPDT[dtype])
    ws = float(oracle.max_wavespeed(shape, u, NPDT[dtype](GAMMA)))
    noflat = oracle.sweep(shape, 0, u, NPDT[dtype](GAMMA), NPDT[dtype](0.8 / ws), flatten=False)
    flat = oracle.sweep(shape, 0, u, NPDT[dtype](GAMMA), NPDT[dtype](0.8 / ws))
    assert not np.array_equal(flat, noflat), "flattening never triggered"
    assert _sweeps(shape, dtype, u, 0.8 / ws, POLICIES[0]) < TOL[dtype]


@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_staged_quadrant_white_noise_and_stiff(cuda, oracle, dtype):
    """Five-decade jumps (flattening active) and the stiffened fluid."""
    from fluidity_b200.workloads import riemann_states
    shape = (96, 80)
    u = oracle.fill_riemann(shape, riemann_states(11, 2), GAMMA, dtype=NPDT[dtype])
    ws = float(oracle.max_wavespeed(shape, u, NPDT[dtype](GAMMA)))
    assert _sweeps(shape, dtype, u, 0.8 / ws, POLICIES[0]) < TOL[dtype]
    us = oracle.prim_to_cons(random_prim(shape, 4, smooth=True, mild=True), GAMMA,
                             dtype=NPDT[dtype])
    with oracle.stiffened(0.613):
        ws = float(oracle.max_wavespeed(shape, us, NPDT[dtype](GAMMA)))
    assert _sweeps(shape, dtype, us, 0.5 / ws, POLICIES[0], p_inf=0.613) < TOL[dtype]


@pytest.mark.parametrize("dtype", ["f64", "f32"])
@pytest.mark.parametrize("shape", [(2048, 2048), (1024, 512), (96, 80)])
def test_loop_and_split_solve_agree(cuda, dtype, shape):
    """The device-resident loop (strips taken dynamically; in FP64 by
    default, and in both dtypes with FLUIDITY_B200_SWEEP=staged, with the
    layouts alternating between sweeps) against fl_split_solve (one strip
    per warp, the caller's layout) replaying the loop's time steps: the
    kernels differ in the x sweep, so the two agree to the parity bars."""
    import torch
    from fluidity_b200.solver import Simulation, SplitSolver
    from fluidity_b200.workloads import riemann_states
    s = SplitSolver(shape, dtype=dtype, gamma=GAMMA)
    a = s.fill_riemann(riemann_states(7, 2))
    u0 = a.clone()
    b = torch.empty_like(a)
    res = 1.0 / shape[0]
    sim = Simulation(s)
    sim.begin(a, b, 0.8, res, 1e30, 2)
    sim.steps(2)
    it, _, done, out = sim.status()
    assert it == 2 and done
    x, y = u0.clone(), torch.empty_like(u0)
    ws = s.max_wavespeed(x).item()
    for _ in range(2):
        if dtype == "f32":
            f32, f64 = np.float32, np.float64
            dt = f32(f64(f32(0.8)) * res / f64(f32(ws)))
            dtdh = float(f32(f64(dt) / res))
        else:
            dtdh = (0.8 * res / ws) / res
        mws = torch.zeros(1, dtype=torch.float64, device="cuda")
        _, x = s.solve(x, y, dtdh, max_ws=mws)
        ws = mws.item()
    torch.cuda.synchronize()
    assert rel_err(out.cpu().numpy(), x.cpu().numpy(), FLOOR[dtype]) < TOL[dtype]


LOOP_CASES = [((96, 80), 0, 0.0), ((100, 36), 3, 0.0), ((64, 48), 0, 0.613),
              ((8, 4), 1, 0.0), ((4, 40), 2, 0.0), ((256, 128), 0, 0.0)]


@pytest.mark.parametrize("dtype", ["f64", "f32"])
@pytest.mark.parametrize("shape,reflect,p_inf", LOOP_CASES,
                         ids=lambda v: "x".join(map(str, v)) if isinstance(v, tuple) else str(v))
def test_loop_matches_oracle_loop(cuda, oracle, shape, dtype, reflect, p_inf):
    """fl_sim_* (device-resident dt; the alternating-layout loop where it
    applies) against the oracle's loop: 12 steps of a smooth field, then the
    iteration count, run time and state.  Whole runs accumulate rounding
    over the steps: FP64 within 1e-10 per cell, FP32 within 1e-4 of the
    component's magnitude."""
    import contextlib
    import torch
    from fluidity_b200.solver import Simulation, SplitSolver
    npdt = NPDT[dtype]
    u = oracle.prim_to_cons(random_prim(shape, 21, smooth=True, mild=True), GAMMA, dtype=npdt)
    ctx = oracle.stiffened(p_inf) if p_inf else contextlib.nullcontext()
    with ctx:
        ref, steps, rt, _ = oracle.simulate(shape, u, npdt(GAMMA), 0.8, 1.0 / shape[0], 1e30, 12,
                                            reflect=reflect)
    s = SplitSolver(shape, dtype=dtype, gamma=GAMMA, boundary_mask=reflect, p_inf=p_inf)
    a = torch.from_numpy(np.ascontiguousarray(u)).to("cuda")
    b = torch.empty_like(a)
    res, it, t = Simulation(s).run(a, b, 0.8, 1.0 / shape[0], 1e30, 12)
    assert it == steps == 12
    assert abs(t - rt) <= (1e-12 if dtype == "f64" else 1e-6) * rt
    bar = (1e-10, 1e-3) if dtype == "f64" else (1e-4, 1.0)
    assert rel_err(res.cpu().numpy(), ref, bar[1]) < bar[0]


def _subset_in_subprocess(mode, path, select):
    env = dict(os.environ, FLUIDITY_B200_SWEEP=mode)
    r = subprocess.run([sys.executable, "-m", "pytest", "-q", "-x", "-p", "no:cacheprovider",
                        os.path.join(ROOT, "tests", path), "-k", select, "-m", "gpu"],
                       cwd=ROOT, env=env, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-2000:]
    assert " passed" in r.stdout


@pytest.mark.parametrize("mode", ["walk", "tile"])
def test_older_2d_kernels_parity_subset(cuda, mode):
    """The register walk and the shared-memory tile kernel stay selectable
    (FLUIDITY_B200_SWEEP=walk|tile, read once per process): the 2-D parity
    subset of test_split_gpu.py in a process of its own."""
    _subset_in_subprocess(mode, "test_split_gpu.py",
                          "quadrant_2d_per_step or (policy_sweeps and 2d) or loop_matches_host "
                          "or dynamic_strips")


def test_staged_x_sweep_parity_subset(cuda):
    """FLUIDITY_B200_SWEEP=staged also takes the transposed staged walk for
    the x sweep: this file's parity cases (not this test) in a process of
    its own."""
    _subset_in_subprocess("staged", "test_staged_gpu.py", "not subset and not older_2d")
