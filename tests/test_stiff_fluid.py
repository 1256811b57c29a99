"""The stiffened fluid (material/stiff_fluid.hpp:38-133) on the split path.

Reference semantics kept here:
- sound speed sqrt(gamma (p + p_inf) / rho) (stiff_fluid.hpp:92-96);
- a state filled from primitives gets e = (p + gamma p_inf) / ((gamma - 1) rho)
  (stiff_fluid.hpp:76-80, state_impl.hpp:136-142);
- the pressure of a conservative state stays (gamma - 1)(E - rho |v|^2 / 2)
  (state_impl.hpp:117-128), so fluxes and flattening see p + gamma p_inf.

The golden fixtures (tests/golden/stiff.npz) are outputs of the reference's own
StiffFluid driven through FaceFlux by oracle/ref_driver.cpp.  CPU tests pin
the oracle's restatement to them bit for bit; GPU tests hold the CUDA path to
the split-path bars: 1e-12 per FP64 sweep (with the pressure's share of the
update in the scale, _stiff_err), 1e-9 for whole runs.
"""
import ctypes as C
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
from make_golden import load  # noqa: E402
from _util import random_prim, rel_err  # noqa: E402

STIFF = load("stiff.npz")
SWEEP_CASES = sorted(k for k, v in STIFF.items() if "dim" in v)
WS_CASES = sorted(k for k in STIFF if k.endswith("__maxws"))
SIM_CASES = sorted(k for k, v in STIFF.items() if "steps" in v)
STAR_CASES = sorted(k for k in STIFF if k.startswith("star_"))


def _shape(c):
    return tuple(int(v) for v in c["shape"])


def _input(c):
    return STIFF[c["src"] + "__maxws"]["u"]


# ---- the oracle against the reference's StiffFluid (CPU) -------------------

def test_fixture_inventory():
    assert len(SWEEP_CASES) == 2 * 4 * (1 + 2 + 3)
    assert len(WS_CASES) == 6 and len(SIM_CASES) == 4 and len(STAR_CASES) == 64


@pytest.mark.parametrize("name", SWEEP_CASES)
def test_oracle_sweep_pinned(oracle, name):
    c = STIFF[name]
    with oracle.stiffened(c["p_inf"]):
        out = oracle.sweep(_shape(c), c["dim"], _input(c), c["gamma"], c["dtdh"], flux=c["flux"],
                           limiter=c["limiter"], recon=c["recon"], reflect=int(c["reflect"]))
    assert np.array_equal(out, c["out"], equal_nan=True)


@pytest.mark.parametrize("name", WS_CASES)
def test_oracle_wavespeed_and_fill_pinned(oracle, name):
    c = STIFF[name]
    with oracle.stiffened(c["p_inf"]):
        assert oracle.max_wavespeed(_shape(c), c["u"], c["gamma"]) == c["ws"]
        assert np.array_equal(oracle.prim_to_cons(c["prim"], c["gamma"]), c["u"])


@pytest.mark.parametrize("name", SIM_CASES)
def test_oracle_simulate_pinned(oracle, name):
    c = STIFF[name]
    shape = _shape(c)
    with oracle.stiffened(c["p_inf"]):
        assert np.array_equal(oracle.fill_riemann(shape, c["states"], c["gamma"]), c["u"])
        out, steps, rt, dts = oracle.simulate(shape, c["u"], c["gamma"], c["cfl"], c["res"],
                                              c["sim_time"], c["max_iters"], flux=c["flux"])
    assert steps == c["steps"] and rt == c["run_time"]
    assert np.array_equal(dts[:steps], c["dts"][:steps])
    assert np.array_equal(out, c["out"])


def test_oracle_mm_star_pinned(oracle):
    """The ghost fluid's two-material star state against the reference's
    Hllc::solve_star_conservative_left for every pairing of the two EOS."""
    for name in STAR_CASES:
        c = STIFF[name]
        got = oracle.mm_star_left(c["ul"], c["ur"], c["gl"], c["il"], c["gr"], c["ir"])
        assert np.array_equal(got, c["star"]), name


def test_stiffened_differs_and_resets(oracle):
    """p_inf changes the sweep (the sound speed enters HLLC), and leaving the
    block restores the ideal gas."""
    shape = (32, 16)
    u = oracle.prim_to_cons(random_prim(shape, 4, smooth=True, mild=True), 1.4)
    ideal = oracle.sweep(shape, 0, u, 1.4, 0.01)
    with oracle.stiffened(0.613):
        stiff = oracle.sweep(shape, 0, u, 1.4, 0.01)
        ws_s = oracle.max_wavespeed(shape, u, 1.4)
    assert not np.array_equal(ideal, stiff)
    assert ws_s > oracle.max_wavespeed(shape, u, 1.4)
    assert np.array_equal(oracle.sweep(shape, 0, u, 1.4, 0.01), ideal)


@pytest.mark.parametrize("gamma,p_inf,needle", [
    (1.0, 0.5, "gamma must exceed 1"), (4.4, -1.0, "p_inf must be finite"),
    (4.4, float("inf"), "p_inf must be finite"), (4.4, float("nan"), "p_inf must be finite"),
])
def test_material_checks(gamma, p_inf, needle):
    """Host-side argument checks of the fl_material entry points; each call
    fails before anything is enqueued, so no device is needed."""
    from fluidity_b200 import capi
    lib = capi.load()
    g = capi.Grid.make((16, 16))
    m = capi.Material(gamma, p_inf)
    fake_in, fake_out = C.c_void_p(256), C.c_void_p(512)   # never dereferenced
    rc = lib.fl_split_sweep_mat(C.byref(g), 0, fake_in, fake_out, C.byref(m), 0.1, 0, 0,
                                None, None)
    assert rc == capi.FL_EINVAL and needle in lib.fl_last_error_string().decode()
    rc = lib.fl_max_wavespeed_mat(C.byref(g), fake_in, C.byref(m), 0, fake_out, None)
    assert rc == capi.FL_EINVAL
    rc = lib.fl_fill_riemann_mat(C.byref(g), fake_in, C.byref(m), 0, fake_out, None)
    assert rc == capi.FL_EINVAL
    assert lib.fl_sim_set_material(None, C.byref(m)) == capi.FL_EINVAL
    assert lib.fl_split_sweep_mat(C.byref(g), 0, fake_in, fake_out, None, 0.1, 0, 0, None,
                                  None) == capi.FL_EINVAL


# ---- the CUDA path (B200) ---------------------------------------------------

def _dev(u, dtype="f64"):
    import torch
    return torch.from_numpy(np.ascontiguousarray(u)).to(
        device="cuda", dtype=torch.float64 if dtype == "f64" else torch.float32)


@pytest.mark.gpu
@pytest.mark.parametrize("name", SWEEP_CASES)
def test_gpu_sweep_matches_reference(cuda, name):
    import torch
    from fluidity_b200.solver import SplitSolver
    c = STIFF[name]
    shape = _shape(c)
    s = SplitSolver(shape, gamma=c["gamma"], p_inf=c["p_inf"], flux=c["flux"],
                    limiter=c["limiter"], recon=c["recon"], boundary_mask=int(c["reflect"]))
    a = _dev(_input(c))
    b = torch.empty_like(a)
    s.sweep(a, b, c["dim"], c["dtdh"])
    assert _stiff_err(b.cpu().numpy(), c["out"], _input(c), c["gamma"], c["dtdh"]) < 1e-12


def _stiff_err(out, ref, u, gamma, dtdh):
    """rel_err's per-cell bar with the pressure term of the update added to
    the denominator.  The state's pressure of a stiffened fluid carries
    gamma p_inf (2100 for p_inf = 343 against p of order 1), so an ulp of it,
    passed into the momentum and energy fluxes and multiplied by dtdh, is far
    above an ulp of the state; the bar measures the kernel against that
    rounding, as 1e-12 of the state does for the ideal gas."""
    D = u.shape[0] - 2
    v2 = sum((u[2 + d] / u[0]) ** 2 for d in range(D))
    p_state = np.max(np.abs((gamma - 1.0) * (u[1] - 0.5 * u[0] * v2)))
    a = np.asarray(out, dtype=np.float64)
    b = np.asarray(ref, dtype=np.float64)
    na, nb = np.isnan(a), np.isnan(b)
    if (na != nb).any():
        return float("inf")                 # NaN in one result only
    a, b = np.where(na, 0.0, a), np.where(nb, 0.0, b)
    scale = np.max(np.abs(b), axis=1, keepdims=True)
    den = np.maximum(np.abs(b), 1e-3 * scale) + dtdh * p_state
    return float(np.max(np.abs(a - b) / den))


@pytest.mark.gpu
@pytest.mark.parametrize("name", WS_CASES)
def test_gpu_wavespeed_and_fill(cuda, name):
    from fluidity_b200.solver import SplitSolver
    c = STIFF[name]
    shape = _shape(c)
    s = SplitSolver(shape, gamma=c["gamma"], p_inf=c["p_inf"])
    ws = s.max_wavespeed(_dev(c["u"])).item()
    assert abs(ws - c["ws"]) <= 1e-14 * c["ws"]


@pytest.mark.gpu
@pytest.mark.parametrize("name", SIM_CASES)
def test_gpu_simulate_matches_reference(cuda, name):
    import torch
    from fluidity_b200.solver import Simulation, SplitSolver
    c = STIFF[name]
    shape = _shape(c)
    s = SplitSolver(shape, gamma=c["gamma"], p_inf=c["p_inf"], flux=c["flux"])
    a = s.fill_riemann(c["states"])
    torch.cuda.synchronize()
    assert np.array_equal(a.cpu().numpy(), c["u"]), "fill differs from State::conservative"
    res, iters, rt = Simulation(s).run(a, torch.empty_like(a), c["cfl"], c["res"],
                                       c["sim_time"], c["max_iters"])
    assert iters == c["steps"]
    assert abs(rt - c["run_time"]) <= 1e-12 * c["run_time"]
    assert rel_err(res.cpu().numpy(), c["out"]) < 1e-9


@pytest.mark.gpu
@pytest.mark.parametrize("shape", [(300,), (70, 45), (20, 13, 11)], ids=["1d", "2d", "3d"])
@pytest.mark.parametrize("flux", ["hllc", "force"])
def test_gpu_f32_sweeps(cuda, oracle, shape, flux):
    """FP32 states: the reference's MUSCL does not compile for float, so the
    FP32 oracle restatement is the checker (1e-5 of each component's scale)."""
    import torch
    from fluidity_b200.solver import SplitSolver
    gamma, p_inf = np.float32(4.4), 0.613
    D = len(shape)
    with oracle.stiffened(p_inf):
        u = oracle.prim_to_cons(random_prim(shape, 40 + D, smooth=True, mild=True), gamma,
                                dtype=np.float32)
        dtdh = np.float32(0.5 / float(oracle.max_wavespeed(shape, u, gamma)))
        for dim in range(D):
            ref = oracle.sweep(shape, dim, u, gamma, dtdh, flux=flux)
            s = SplitSolver(shape, dtype="f32", gamma=float(gamma), p_inf=p_inf, flux=flux)
            a = _dev(u, "f32")
            b = torch.empty_like(a)
            s.sweep(a, b, dim, float(dtdh))
            assert rel_err(b.cpu().numpy(), ref, 1.0) < 1e-5


@pytest.mark.gpu
def test_gpu_zero_p_inf_is_the_ideal_gas(cuda):
    """The fl_material entry points with p_inf = 0 equal the gamma-only ones
    bit for bit."""
    import torch
    from fluidity_b200 import capi
    from fluidity_b200.solver import SplitSolver
    shape = (96, 64)
    s = SplitSolver(shape, gamma=1.4)
    st = np.array([[1.0, 1.0, 0.0, 0.0], [0.5, 0.4, 0.3, 0.0],
                   [0.8, 0.6, 0.0, -0.2], [0.125, 0.1, 0.1, 0.1]])
    a = s.fill_riemann(st)
    b0, b1 = torch.empty_like(a), torch.empty_like(a)
    ws0 = torch.zeros(1, dtype=torch.float64, device="cuda")
    ws1 = torch.zeros_like(ws0)
    s.sweep(a, b0, 1, 0.3, max_ws=ws0)
    m = capi.Material(1.4, 0.0)
    rc = s.lib.fl_split_sweep_mat(C.byref(s.grid), 1, C.c_void_p(a.data_ptr()),
                                  C.c_void_p(b1.data_ptr()), C.byref(m), 0.3, s.policy, 0,
                                  C.c_void_p(ws1.data_ptr()), None)
    capi.check(rc, s.lib)
    torch.cuda.synchronize()
    assert torch.equal(b0, b1) and torch.equal(ws0, ws1)


# ---- two materials: gas and a stiffened fluid -------------------------------

def _mm_initial(spec, p_infs, dtype):
    from oracle import oracle as O
    n = spec["nx"] * spec["ny"]
    g0, g1 = spec["gammas"]
    allin = -np.ones(n)
    u0 = O.mm_set_states(np.zeros((4, n), dtype=dtype), allin, spec["ambient"], g0, p_infs[0])
    u0 = O.mm_set_states(u0, spec["shock_phi"], spec["shocked"], g0, p_infs[0])
    u1 = O.mm_set_states(np.zeros((4, n), dtype=dtype), allin, spec["bubble"], g1, p_infs[1])
    return u0, u1


def _mm_relerr(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    scale = np.maximum(np.max(np.abs(b), axis=1, keepdims=True), 1e-3 * np.max(np.abs(b)))
    return float(np.max(np.abs(a - b) / scale))


P_INFS = (0.0, 0.613)     # ambient gas | stiffened bubble


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_gpu_mm_stiff_ghost_bit_exact(cuda, oracle, dtype):
    """Shock-bubble data whose bubble is a stiffened fluid: set_states and
    the ghost pass (GFM star states with each side's sound speed, then the
    extrapolation) match the oracle bit for bit."""
    import torch
    from fluidity_b200.multimaterial import MultiMaterial
    from fluidity_b200.workloads import shock_bubble
    spec = shock_bubble(6, nx=128, ny=64, width=2.0)
    npdt = np.float32 if dtype == "f32" else np.float64
    u0, u1 = _mm_initial(spec, P_INFS, npdt)
    mm = MultiMaterial.shock_bubble(spec, dtype=dtype, p_infs=P_INFS)
    got0, got1 = (t.cpu().numpy() for t in mm.states())
    assert np.array_equal(got0, u0) and np.array_equal(got1, u1)
    w0, w1 = oracle.mm_ghost(spec["nx"], spec["ny"], spec["h"], spec["gammas"], u0, u1,
                             spec["phi0"], spec["phi1"], p_infs=P_INFS)
    mm.ghost()
    g0, g1 = (t.cpu().numpy() for t in mm.states())
    assert np.array_equal(g0, w0) and np.array_equal(g1, w1)
    i0, i1 = oracle.mm_ghost(spec["nx"], spec["ny"], spec["h"], spec["gammas"], u0, u1,
                             spec["phi0"], spec["phi1"])
    assert not np.array_equal(w1, i1), "p_inf never reached the star states"


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_gpu_mm_stiff_steps(cuda, oracle, dtype):
    """Four steps of the two-material loop with a stiffened bubble against the
    oracle loop (1e-7 FP64, 1e-4 FP32 of each component's scale)."""
    import torch
    from fluidity_b200.multimaterial import MultiMaterial
    from fluidity_b200.workloads import shock_bubble
    spec = shock_bubble(7, nx=96, ny=48, width=2.0)
    npdt = np.float32 if dtype == "f32" else np.float64
    u0, u1 = _mm_initial(spec, P_INFS, npdt)
    mm = MultiMaterial.shock_bubble(spec, dtype=dtype, p_infs=P_INFS)
    nsteps, every = 4, 2
    mm.begin(cfl=0.6, sim_time=1e9, max_iters=nsteps, reinit_every=every)
    mm.steps(nsteps)
    it, rt, done = mm.status()
    assert it == nsteps and done
    p0, p1 = spec["phi0"], spec["phi1"]
    t = 0.0
    for k in range(nsteps):
        u0, u1, p0, p1, dt = oracle.mm_step(spec["nx"], spec["ny"], spec["h"], spec["gammas"],
                                            0.6, u0, u1, p0, p1, reinit=((k + 1) % every == 0),
                                            p_infs=P_INFS)
        t += dt
    assert abs(rt - t) < 1e-9 * t
    g0, g1 = (x.cpu().numpy() for x in mm.states())
    tol = 1e-4 if dtype == "f32" else 1e-7
    assert _mm_relerr(g0, u0) < tol and _mm_relerr(g1, u1) < tol


def test_mm_material_checks():
    from fluidity_b200 import capi
    lib = capi.load()
    bad = (capi.Material * 2)(capi.Material(1.4, 0.0), capi.Material(4.4, -0.5))
    assert lib.fl_mm_set_materials(None, bad) == capi.FL_EINVAL
    g = capi.Grid.make((16, 16))
    fake = C.c_void_p(256)                                     # never dereferenced
    prim = (C.c_double * 4)(1.0, 1.0, 0.0, 0.0)
    assert lib.fl_mm_set_states_mat(C.byref(g), 0, fake, fake, prim, C.byref(bad[1]),
                                    None) == capi.FL_EINVAL
