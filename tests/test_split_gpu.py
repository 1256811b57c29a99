"""Parity of the CUDA split-solver step (through the C ABI) with the CPU
oracle and with the golden fixtures computed by the reference's functors.

Tolerances, per cell and per step (see _util.rel_err):
* FP64: 1e-12 relative to the cell's value, floored at 1e-3 of the
  component's largest magnitude (near-zero momenta are differences of O(p)
  flux terms, so their own size is no yardstick);
* FP32: 1e-5 relative to the component's largest magnitude.  FP32 rounding
  (6e-8) is amplified by the flux differences of the update, so a per-value
  relative bar would measure cancellation, not the kernel.
The CUDA build contracts multiply-adds into FMA and forms velocities with one
reciprocal per state, so results differ from the reference by rounding only.
"""
import ctypes as C
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
from make_golden import load  # noqa: E402
from _util import random_prim, rel_err  # noqa: E402

pytestmark = pytest.mark.gpu

GAMMA = 1.4
TOL = {"f64": 1e-12, "f32": 1e-5}
FLOOR = {"f64": 1e-3, "f32": 1.0}


def err(a, b, dtype):
    return rel_err(a, b, FLOOR[dtype])
NPDT = {"f64": np.float64, "f32": np.float32}


def to_dev(u, dtype, pitch=None):
    import torch
    D2, cells = u.shape
    pitch = cells if pitch is None else pitch
    t = torch.zeros((D2, pitch), dtype=torch.float64 if dtype == "f64" else torch.float32,
                    device="cuda")
    t[:, :cells] = torch.from_numpy(np.ascontiguousarray(u, dtype=NPDT[dtype]))
    return t


def to_host(t, cells):
    return t[:, :cells].cpu().numpy()


def gpu_sweep(shape, dim, u, dtdh, dtype="f64", pitch=None, want_ws=False, **pol):
    import torch
    from fluidity_b200.solver import SplitSolver
    s = SplitSolver(shape, dtype=dtype, gamma=GAMMA, pitch=pitch,
                    flux=pol.get("flux", "hllc"), limiter=pol.get("limiter", "vanleer"),
                    recon=pol.get("recon", "muscl"), boundary_mask=pol.get("reflect", 0),
                    flatten=pol.get("flatten", True))
    a = to_dev(u, dtype, s.grid.pitch)
    b = torch.empty_like(a)
    ws = torch.zeros(1, dtype=torch.float64, device="cuda") if want_ws else None
    s.sweep(a, b, dim, dtdh, max_ws=ws)
    torch.cuda.synchronize()
    out = to_host(b, int(np.prod(shape)))
    return (out, float(ws.item())) if want_ws else out


# ---- golden fixtures (reference functors) ---------------------------------

SWEEPS = load("sweeps.npz")
SIMS = load("simulate.npz")


@pytest.mark.parametrize("name", sorted(k for k in SWEEPS if "maxws" not in k))
def test_sweep_matches_reference_golden(cuda, name):
    c = SWEEPS[name]
    shape = tuple(int(v) for v in c["shape"])
    out = gpu_sweep(shape, int(c["dim"]), c["u"], c["dtdh"], flux=c["flux"],
                    limiter=c["limiter"], recon=c["recon"], reflect=int(c["reflect"]))
    ref = c["out"]
    finite = np.isfinite(ref).all(axis=0)
    # cells the reference blows up (white-noise inputs) must blow up here too
    assert not np.isfinite(out[:, ~finite]).all(axis=0).any()
    assert rel_err(out[:, finite], ref[:, finite]) < TOL["f64"]


@pytest.mark.parametrize("name", sorted(k for k in SWEEPS if "maxws" in k))
def test_max_wavespeed_matches_reference_golden(cuda, name):
    import torch
    from fluidity_b200.solver import SplitSolver
    c = SWEEPS[name]
    shape = tuple(int(v) for v in c["shape"])
    s = SplitSolver(shape, gamma=GAMMA)
    ws = s.max_wavespeed(to_dev(c["u"], "f64")).item()
    assert abs(ws - c["ws"]) <= 1e-14 * c["ws"]


@pytest.mark.parametrize("name", sorted(SIMS))
def test_simulate_matches_reference_golden(cuda, name):
    """Whole device-resident runs against the reference's own loop."""
    import torch
    from fluidity_b200.solver import Simulation, SplitSolver
    c = SIMS[name]
    shape = tuple(int(v) for v in c["shape"])
    s = SplitSolver(shape, gamma=GAMMA, flux=c["flux"], limiter=c["limiter"],
                    recon=c["recon"], boundary_mask=int(c["reflect"]))
    a = s.fill_riemann(c["states"])
    torch.cuda.synchronize()
    assert np.array_equal(to_host(a, a.shape[1]), c["u"]), "initial state differs"
    b = torch.empty_like(a)
    sim = Simulation(s)
    res, iters, rt = sim.run(a, b, c["cfl"], c["res"], c["sim_time"], c["max_iters"])
    assert iters == c["steps"]
    assert abs(rt - c["run_time"]) <= 1e-12 * c["run_time"]
    # whole runs accumulate FMA rounding over every step: 1e-9 here; the
    # per-step bar of 1e-12 is checked step by step below
    assert rel_err(to_host(res, res.shape[1]), c["out"]) < 1e-9


# ---- step-by-step parity with the oracle ----------------------------------

@pytest.mark.parametrize("dtype", ["f64", "f32"])
@pytest.mark.parametrize("seed", [0, 1, 2])
def test_tube_per_step_parity(cuda, oracle, dtype, seed):
    """1-D N=400 Riemann tube (HLLC, van Leer, CFL 0.9, to t = 0.25/max ws):
    at every step the GPU step applied to the oracle's state matches the
    oracle's next state."""
    import torch
    from fluidity_b200.solver import SplitSolver
    from fluidity_b200.workloads import riemann_states
    shape = (400,)
    npdt = NPDT[dtype]
    u = oracle.fill_riemann(shape, riemann_states(seed, 1), GAMMA, dtype=npdt)
    s = SplitSolver(shape, dtype=dtype, gamma=GAMMA)
    t_end = 0.25 / float(oracle.max_wavespeed(shape, u, npdt(GAMMA)))
    t = 0.0
    steps = 0
    worst = 0.0
    a = torch.empty((3, 400), dtype=torch.float64 if dtype == "f64" else torch.float32,
                    device="cuda")
    b = torch.empty_like(a)
    while t < t_end and steps < 2000:
        ws = float(oracle.max_wavespeed(shape, u, npdt(GAMMA)))
        dt = npdt(0.9 * (1.0 / 400) / ws)
        dtdh = npdt(float(dt) / (1.0 / 400))
        nxt = oracle.sweep(shape, 0, u, npdt(GAMMA), dtdh)
        a.copy_(torch.from_numpy(u))
        s.sweep(a, b, 0, float(dtdh))
        worst = max(worst, err(b.cpu().numpy(), nxt, dtype))
        u = nxt
        t += float(dt)
        steps += 1
    assert steps > 50
    assert worst < TOL[dtype], f"worst per-step error {worst:.3e} over {steps} steps"


@pytest.mark.parametrize("dtype", ["f64", "f32"])
@pytest.mark.parametrize("flux", ["hllc", "force"])
def test_quadrant_2d_per_step_parity(cuda, oracle, dtype, flux):
    """2-D four-quadrant problem, 96 x 80 (partial tiles in both dims): each
    step's x and y sweeps against the oracle, ten steps, CFL 0.8."""
    import torch
    from fluidity_b200.solver import SplitSolver
    from fluidity_b200.workloads import riemann_states
    shape = (96, 80)
    npdt = NPDT[dtype]
    u = oracle.fill_riemann(shape, riemann_states(11, 2), GAMMA, dtype=npdt)
    s = SplitSolver(shape, dtype=dtype, flux=flux, gamma=GAMMA)
    res = 1.0 / 96
    worst = 0.0
    for _ in range(10):
        ws = float(oracle.max_wavespeed(shape, u, npdt(GAMMA)))
        dt = npdt(0.8 * res / ws)
        dtdh = npdt(float(dt) / res)
        mid = oracle.sweep(shape, 0, u, npdt(GAMMA), dtdh, flux=flux)
        nxt = oracle.sweep(shape, 1, mid, npdt(GAMMA), dtdh, flux=flux)
        a = to_dev(u, dtype)
        b = torch.empty_like(a)
        s.sweep(a, b, 0, float(dtdh))
        worst = max(worst, err(b.cpu().numpy(), mid, dtype))
        a.copy_(torch.from_numpy(mid))
        s.sweep(a, b, 1, float(dtdh))
        worst = max(worst, err(b.cpu().numpy(), nxt, dtype))
        u = nxt
    assert worst < TOL[dtype], f"worst per-step error {worst:.3e}"


# ---- policy coverage on smooth data --------------------------------------

POLICIES = [
    ("hllc", "vanleer", "muscl", True), ("force", "vanleer", "muscl", True),
    ("lf", "superbee", "muscl", True), ("richtmyer", "vanleer", "muscl", True),
    ("hllc", "superbee", "basic", True), ("hllc", "vanleer", "muscl", False),
]


@pytest.mark.parametrize("shape", [(300,), (70, 45), (20, 13, 11)], ids=["1d", "2d", "3d"])
@pytest.mark.parametrize("dtype", ["f64", "f32"])
@pytest.mark.parametrize("pol", POLICIES, ids=lambda p: "-".join(str(x) for x in p))
def test_policy_sweeps(cuda, oracle, shape, dtype, pol):
    flux, lim, recon, flatten = pol
    npdt = NPDT[dtype]
    D = len(shape)
    u = oracle.prim_to_cons(random_prim(shape, 7 + D, smooth=True, mild=True),
                            GAMMA).astype(npdt)
    ws = float(oracle.max_wavespeed(shape, u, npdt(GAMMA)))
    dtdh = npdt(0.5 / ws)
    for dim in range(D):
        for reflect in (0, (1 << D) - 1):
            ref = oracle.sweep(shape, dim, u, npdt(GAMMA), dtdh, flux=flux, limiter=lim,
                               recon=recon, flatten=flatten, reflect=reflect)
            out = gpu_sweep(shape, dim, u, float(dtdh), dtype=dtype, flux=flux, limiter=lim,
                            recon=recon, flatten=flatten, reflect=reflect)
            assert err(out, ref, dtype) < TOL[dtype], (dim, reflect)


@pytest.mark.parametrize("shape", [(4, 5, 6), (33, 4, 7), (7, 9, 70), (26, 26, 5)],
                         ids=lambda s: "x".join(map(str, s)))
@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_3d_walk_shapes(cuda, oracle, shape, dtype):
    """The 3-D walk at the minimum extent (4), at extents that split a warp's
    columns or a strip's rows unevenly, and with reflective ends in every
    dimension; each sweep with its fused wavespeed against the oracle."""
    npdt = NPDT[dtype]
    u = oracle.prim_to_cons(random_prim(shape, 50 + shape[0], smooth=True, mild=True),
                            GAMMA).astype(npdt)
    ws = float(oracle.max_wavespeed(shape, u, npdt(GAMMA)))
    dtdh = npdt(0.5 / ws)
    for reflect in (0, 7):
        for dim in range(3):
            ref = oracle.sweep(shape, dim, u, npdt(GAMMA), dtdh, reflect=reflect)
            out, got_ws = gpu_sweep(shape, dim, u, float(dtdh), dtype=dtype, reflect=reflect,
                                    want_ws=True)
            assert err(out, ref, dtype) < TOL[dtype], (dim, reflect)
            # the fused maximum against the oracle's maximum of the same output
            ref_ws = float(oracle.max_wavespeed(shape, out.astype(npdt), npdt(GAMMA)))
            assert abs(got_ws - ref_ws) <= (1e-14 if dtype == "f64" else 1e-6) * ref_ws


@pytest.mark.parametrize("shape", [(100001,), (317, 211), (37, 29, 23)],
                         ids=lambda s: "x".join(map(str, s)))
@pytest.mark.parametrize("where", ["first", "middle", "last"])
def test_max_wavespeed_odd_sizes(cuda, oracle, shape, where):
    """The CFL maximum (the reference's set_wavespeeds + max_element,
    algorithm_tests_device.cu:42-77 tests its reduce on 100001 values) over
    sizes that fill no block evenly, with the largest wavespeed planted at the
    first, a middle or the last cell."""
    from fluidity_b200.solver import SplitSolver
    D = len(shape)
    cells = int(np.prod(shape))
    prim = random_prim(shape, 60 + D, smooth=True, mild=True)   # wavespeeds below 5
    k = {"first": 0, "middle": cells // 2 + 7, "last": cells - 1}[where]
    prim[2:, k] = 40.0                         # the fastest cell
    u = oracle.prim_to_cons(prim, GAMMA)
    s = SplitSolver(shape, gamma=GAMMA)
    ws = s.max_wavespeed(to_dev(u, "f64")).item()
    ref = float(oracle.max_wavespeed(shape, u, GAMMA))
    assert abs(ws - ref) <= 1e-14 * ref
    assert ref > 40.0                          # max_d |u_d| + a of the planted cell


def test_flattening_active_parity(cuda, oracle):
    """A compressive front smeared over a few cells (a sharp jump has one zero
    one-sided difference, so the limiter already kills its slope), oblique so
    that chi < 1 in both dimensions."""
    shape = (64, 48)
    prim = np.zeros((4, 64 * 48))
    x = np.tile(np.arange(64), 48)
    y = np.repeat(np.arange(48), 64)
    w = np.clip((x + y - 50) / 4.0, 0.0, 1.0)      # 0 behind, 1 ahead, 4-cell ramp
    prim[0] = 3.0 + (0.5 - 3.0) * w
    prim[1] = 20.0 + (1.0 - 20.0) * w
    prim[2] = 1.0 + (-0.5 - 1.0) * w
    prim[3] = 1.0 + (-0.5 - 1.0) * w
    u = oracle.prim_to_cons(prim, GAMMA)
    ws = oracle.max_wavespeed(shape, u, GAMMA)
    for dim in (0, 1):
        ref = oracle.sweep(shape, dim, u, GAMMA, 0.8 / ws)
        noflat = oracle.sweep(shape, dim, u, GAMMA, 0.8 / ws, flatten=False)
        assert not np.array_equal(ref, noflat), "flattening never triggered"
        out = gpu_sweep(shape, dim, u, 0.8 / ws)
        assert rel_err(out, ref) < TOL["f64"]


def test_pitch_padding(cuda, oracle):
    """Component planes with a pitch larger than the cell count."""
    shape = (50, 30)
    u = oracle.prim_to_cons(random_prim(shape, 3, smooth=True, mild=True), GAMMA)
    ref = oracle.sweep(shape, 1, u, GAMMA, 0.001)
    out = gpu_sweep(shape, 1, u, 0.001, pitch=1600)
    assert rel_err(out, ref) < TOL["f64"]


def test_fused_wavespeed_of_output(cuda, oracle):
    shape = (128, 64)
    u = oracle.prim_to_cons(random_prim(shape, 5, smooth=True, mild=True), GAMMA)
    out, ws = gpu_sweep(shape, 1, u, 0.002, want_ws=True)
    ref = oracle.max_wavespeed(shape, out, GAMMA)
    assert abs(ws - ref) <= 1e-14 * ref


# ---- the device-resident loop ---------------------------------------------

def test_loop_matches_host_loop(cuda, oracle):
    """fl_sim_* (device-resident dt) against the oracle's time loop, 2-D."""
    import torch
    from fluidity_b200.solver import Simulation, SplitSolver
    from fluidity_b200.workloads import riemann_states
    shape = (64, 64)
    u = oracle.fill_riemann(shape, riemann_states(3, 2), GAMMA)
    ref, steps, rt, dts = oracle.simulate(shape, u, GAMMA, 0.8, 1 / 64, 1e30, 15)
    s = SplitSolver(shape, gamma=GAMMA)
    a = to_dev(u, "f64")
    b = torch.empty_like(a)
    sim = Simulation(s)
    sim.begin(a, b, 0.8, 1 / 64, 1e30, 15)
    sim.steps(7)
    it, t, done, _ = sim.status()
    assert it == 7 and not done
    sim.steps(8)
    it, t, done, res = sim.status()
    assert it == 15 and done
    assert abs(t - rt) <= 1e-12 * rt
    assert rel_err(res.cpu().numpy(), ref) < 1e-10


@pytest.mark.parametrize("shape", [(257,), (65, 33), (17, 12, 10)])
def test_reflective_box_conserves(cuda, shape):
    """Reflective walls in every dimension, gas initially at rest with
    moderate contrasts: the flow at the walls stays subsonic, the HLLC star
    speed at a wall is exactly zero and no mass or energy leaves.  (Under
    supersonic inflow the PVRS wave estimate puts S_L > 0 and HLLC returns
    the ghost's own flux, so the reference's walls then pass mass.)"""
    import torch
    from fluidity_b200.solver import Simulation, SplitSolver
    from fluidity_b200.workloads import riemann_states
    D = len(shape)
    s = SplitSolver(shape, gamma=GAMMA, boundary_mask=(1 << D) - 1)
    st = riemann_states(40 + D, D)
    st[:, 0] = np.clip(st[:, 0], 0.5, 2.0)
    st[:, 1] = np.clip(st[:, 1], 0.5, 5.0)
    st[:, 2:] = 0.0
    a = s.fill_riemann(st)
    m0 = a[0].sum().item()
    e0 = a[1].sum().item()
    b = torch.empty_like(a)
    res, it, _ = Simulation(s).run(a, b, 0.6, 1.0 / shape[0], 1e30, 40)
    assert it == 40
    assert abs(res[0].sum().item() - m0) <= 1e-12 * m0
    assert abs(res[1].sum().item() - e0) <= 1e-12 * e0


def test_sim_time_stop_and_result_buffer(cuda, oracle):
    import torch
    from fluidity_b200.solver import Simulation, SplitSolver
    from fluidity_b200.workloads import riemann_states
    shape = (400,)
    u = oracle.fill_riemann(shape, riemann_states(0, 1), GAMMA)
    t_end = 0.1 / oracle.max_wavespeed(shape, u, GAMMA)
    ref, steps, rt, _ = oracle.simulate(shape, u, GAMMA, 0.9, 1 / 400, t_end, 10 ** 9)
    s = SplitSolver(shape, gamma=GAMMA)
    a = to_dev(u, "f64")
    b = torch.empty_like(a)
    res, it, t = Simulation(s).run(a, b, 0.9, 1 / 400, t_end, 10 ** 9)
    assert it == steps
    assert (res.data_ptr() == b.data_ptr()) == (steps % 2 == 1)
    assert rel_err(res.cpu().numpy(), ref) < 1e-10


def test_nan_state_reports_enan(cuda):
    import torch
    from fluidity_b200 import capi
    from fluidity_b200.solver import Simulation, SplitSolver
    s = SplitSolver((64,), gamma=GAMMA)
    a = s.fill_riemann(np.array([[1.0, 1.0, 0.0], [0.125, 0.1, 0.0]]))
    a[1, 10] = float("nan")
    b = torch.empty_like(a)
    with pytest.raises(capi.FlError) as e:
        Simulation(s).run(a, b, 0.9, 1 / 64, 1.0, 100)
    assert e.value.code == capi.FL_ENAN


@pytest.mark.parametrize("where", [(100, 77), (0, 0), (255, 255), (31, 130)])
def test_nan_anywhere_reports_enan(cuda, where):
    """A NaN in one cell of a 2-D state stops the loop with FL_ENAN whatever
    position it has in the kernels' fold order (initial wavespeed, fused
    per-lane, warp and CTA maxima)."""
    import torch
    from fluidity_b200 import capi
    from fluidity_b200.solver import Simulation, SplitSolver
    s = SplitSolver((256, 256), gamma=GAMMA)
    a = s.fill_riemann(np.array([[1.0, 1.0, 0.0, 0.0], [0.5, 0.4, 0.1, 0.0],
                                 [0.8, 0.6, 0.0, 0.1], [0.3, 0.3, 0.0, 0.0]]))
    a[1, where[1] * 256 + where[0]] = float("nan")
    b = torch.empty_like(a)
    with pytest.raises(capi.FlError) as e:
        Simulation(s).run(a, b, 0.8, 1 / 256, 1e30, 2)
    assert e.value.code == capi.FL_ENAN


def test_split_solve_swaps_like_reference(cuda, oracle):
    import torch
    from fluidity_b200.solver import SplitSolver
    for shape in [(40,), (40, 24), (12, 10, 8)]:
        u = oracle.prim_to_cons(random_prim(shape, 1, smooth=True, mild=True), GAMMA)
        s = SplitSolver(shape, gamma=GAMMA)
        a = to_dev(u, "f64")
        b = torch.empty_like(a)
        i, o = s.solve(a, b, 0.001)
        ref = u
        for d in range(len(shape)):
            ref = oracle.sweep(shape, d, ref, GAMMA, 0.001)
        # the reference leaves the result in `out` after swapping iterators
        assert o.data_ptr() == (a if len(shape) % 2 == 0 else b).data_ptr()
        assert rel_err(o.cpu().numpy(), ref) < TOL["f64"]


def test_fill_riemann_bit_exact(cuda, oracle):
    from fluidity_b200.solver import SplitSolver
    from fluidity_b200.workloads import riemann_states
    for shape in [(400,), (97, 50), (9, 8, 7)]:
        D = len(shape)
        st = riemann_states(5, D)
        for dtype in ("f64", "f32"):
            s = SplitSolver(shape, dtype=dtype, gamma=GAMMA)
            got = s.fill_riemann(st).cpu().numpy()
            ref = oracle.fill_riemann(shape, st, GAMMA, dtype=NPDT[dtype])
            assert np.array_equal(got, ref)


def test_aos_soa_round_trip(cuda):
    import torch
    from fluidity_b200 import capi
    lib = capi.load()
    g = capi.Grid.make((33, 17), pitch=600)
    soa = torch.randn(4, 600, dtype=torch.float64, device="cuda")
    aos = torch.empty(33 * 17 * 4, dtype=torch.float64, device="cuda")
    back = torch.zeros_like(soa)
    capi.check(lib.fl_soa_to_aos(C.byref(g), 0, C.c_void_p(soa.data_ptr()),
                                 C.c_void_p(aos.data_ptr()), None))
    capi.check(lib.fl_aos_to_soa(C.byref(g), 0, C.c_void_p(aos.data_ptr()),
                                 C.c_void_p(back.data_ptr()), None))
    torch.cuda.synchronize()
    n = 33 * 17
    assert torch.equal(aos.view(n, 4).t(), soa[:, :n])
    assert torch.equal(back[:, :n], soa[:, :n])


def test_repeatable_bitwise(cuda, oracle):
    import torch
    from fluidity_b200.solver import Simulation, SplitSolver
    from fluidity_b200.workloads import riemann_states
    s = SplitSolver((200, 150), gamma=GAMMA, flux="force")
    outs = []
    for _ in range(2):
        a = s.fill_riemann(riemann_states(9, 2))
        b = torch.empty_like(a)
        res, _, _ = Simulation(s).run(a, b, 0.8, 1 / 200, 1e30, 12)
        outs.append(res.clone())
    assert torch.equal(outs[0], outs[1])


@pytest.mark.parametrize("seed", [0, 1])
def test_f32_l1_against_f64_oracle(cuda, oracle, seed):
    """FP32 run of the 1-D tube against the FP64 oracle: the L1 error of each
    component, relative to the component's L1 norm, is reported and bounded."""
    import torch
    from fluidity_b200.solver import Simulation, SplitSolver
    from fluidity_b200.workloads import riemann_states
    shape = (400,)
    st = riemann_states(seed, 1)
    u64 = oracle.fill_riemann(shape, st, GAMMA)
    t_end = 0.25 / oracle.max_wavespeed(shape, u64, GAMMA)
    ref, steps, _, _ = oracle.simulate(shape, u64, GAMMA, 0.9, 1 / 400, t_end, 10 ** 9)
    s = SplitSolver(shape, dtype="f32", gamma=GAMMA)
    a = s.fill_riemann(st)
    b = torch.empty_like(a)
    res, it, _ = Simulation(s).run(a, b, 0.9, 1 / 400, t_end, 10 ** 9)
    got = res.double().cpu().numpy()
    l1 = np.sum(np.abs(got - ref), axis=1) / np.sum(np.abs(ref), axis=1)
    print(f"seed {seed}: FP32 steps {it} (FP64 {steps}), relative L1 per component {l1}")
    assert abs(it - steps) <= 2
    assert np.all(l1 < 1e-4)


@pytest.mark.parametrize("dtype", ["f64", "f32"])
@pytest.mark.parametrize("shape", [(2048, 2048), (1024, 1024), (700, 300)])
def test_dynamic_strips_equal_static_grid(cuda, dtype, shape):
    """Three paths over two steps, the static ones replaying the loop's own
    time steps: the device-resident loop (strips taken dynamically; 64-row
    strips at 2048^2, shortened to 32 rows where 64-row strips cannot fill
    the GPU), fl_split_solve_ws (the drop-in step with a workspace, strips
    taken dynamically too) and fl_split_solve (one strip per warp).
    * fl_split_solve_ws against fl_split_solve: the schedule decides only
      which warp computes a cell, so FP64 agrees bit for bit.  The register
      walk's two schedules are separately inlined copies of the strip code,
      which the compiler contracts differently in FP32 (6e-7 relative
      measured), so FP32 agrees to rounding.
    * the loop against fl_split_solve_ws: with the register walk for both
      (FLUIDITY_B200_SWEEP=walk) bit for bit; by default the FP64 loop
      alternates layouts and sweeps x with the staged walk while the drop-in
      step sweeps x with the register walk, and the two agree to the FP64
      parity bar."""
    import torch
    from fluidity_b200.solver import Simulation, SplitSolver
    from fluidity_b200.workloads import riemann_states
    s = SplitSolver(shape, dtype=dtype, gamma=GAMMA)
    s_static = SplitSolver(shape, dtype=dtype, gamma=GAMMA, workspace=False)
    a = s.new_state()
    s.fill_riemann(riemann_states(7, 2), out=a)
    u0 = a.clone()
    b = torch.empty_like(a)
    res = 1.0 / shape[0]
    sim = Simulation(s)
    sim.begin(a, b, 0.8, res, 1e30, 2)
    sim.steps(2)
    it, _, done, out = sim.status()
    assert it == 2 and done
    outs = []
    for solver in (s, s_static):
        x, y = u0.clone(), torch.empty_like(u0)
        ws = solver.max_wavespeed(x).item()
        for _ in range(2):
            # the time step as the device computes it (finalize_control)
            if dtype == "f32":
                f32, f64 = np.float32, np.float64
                dt = f32(f64(f32(0.8)) * res / f64(f32(ws)))
                dtdh = float(f32(f64(dt) / res))
            else:
                dtdh = (0.8 * res / ws) / res
            mws = torch.zeros(1, dtype=torch.float64, device="cuda")
            _, x = solver.solve(x, y, dtdh, max_ws=mws)      # 2-D: the result returns to x
            ws = mws.item()
        torch.cuda.synchronize()
        outs.append(x)
    dyn, static = outs

    def close(p, q, bar=1e-5):
        d = (p.double() - q.double()).abs()
        return (d / q.double().abs().clamp_min(1.0)).max().item() < bar

    if dtype == "f64":
        assert torch.equal(dyn, static)
    else:
        assert close(dyn, static)
    if os.environ.get("FLUIDITY_B200_SWEEP") == "walk":
        assert torch.equal(out, dyn)
    elif dtype == "f64":
        assert rel_err(out.cpu().numpy(), dyn.cpu().numpy()) < TOL["f64"]
    else:
        assert close(out, dyn)


def test_workspace_bytes_and_checks(cuda):
    """fl_workspace_bytes: a 256-byte head, plus one value per cell in 3-D;
    a workspace that is not 256-byte aligned is refused before any launch."""
    import ctypes as C
    import torch
    from fluidity_b200 import capi
    from fluidity_b200.solver import SplitSolver
    lib = capi.load()
    for shape, dtype, want in [((64, 48), "f64", 256), ((10, 8, 6), "f64", 256 + 3840),
                               ((10, 8, 6), "f32", 256 + 2048), ((400,), "f32", 256)]:
        s = SplitSolver(shape, dtype=dtype, gamma=GAMMA)
        assert lib.fl_workspace_bytes(C.byref(s.grid), s.policy) == want
    s = SplitSolver((64, 48), gamma=GAMMA)
    a = s.fill_riemann(np.array([[1.0, 1.0, 0.0, 0.0], [0.5, 0.4, 0.1, 0.0],
                                 [0.8, 0.6, 0.0, 0.1], [0.3, 0.3, 0.0, 0.0]]))
    b = torch.empty_like(a)
    raw = torch.zeros(1024, dtype=torch.uint8, device="cuda")
    rc = lib.fl_split_sweep_ws(C.byref(s.grid), 0, C.c_void_p(a.data_ptr()),
                               C.c_void_p(b.data_ptr()), C.byref(s.material), 0.001, s.policy, 0,
                               None, C.c_void_p(raw.data_ptr() + 8), None)
    assert rc == capi.FL_EINVAL
    assert s.workspace_status() == 0


@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_workspace_3d_walk_and_tile_match_oracle(cuda, oracle, dtype):
    """3-D sweeps: with a workspace the register walk (its flattening plane
    in the workspace), without one the tile kernel; both at the parity bars,
    and the workspace reused across calls without being cleared."""
    import torch
    from fluidity_b200.solver import SplitSolver
    shape = (20, 13, 11)
    npdt = NPDT[dtype]
    u = oracle.prim_to_cons(random_prim(shape, 3, smooth=True, mild=True), GAMMA, dtype=npdt)
    ws = float(oracle.max_wavespeed(shape, u, npdt(GAMMA)))
    dtdh = npdt(0.5 / ws)
    for workspace in (True, False):
        s = SplitSolver(shape, dtype=dtype, gamma=GAMMA, workspace=workspace)
        for dim in (0, 1, 2, 0):
            ref = oracle.sweep(shape, dim, u, npdt(GAMMA), dtdh)
            a = to_dev(u, dtype)
            b = torch.empty_like(a)
            s.sweep(a, b, dim, float(dtdh))
            torch.cuda.synchronize()
            assert err(b.cpu().numpy(), ref, dtype) < TOL[dtype], (workspace, dim)
