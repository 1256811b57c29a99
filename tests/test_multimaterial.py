"""Two-material ghost-fluid path: oracle properties on CPU, then the CUDA
kernels and the step loop against the oracle on the same seeded inputs.

Reference: ghost_fluid/riemann_ghost_fluid.hpp (RiemannGFM<3>),
ghost_fluid/ghost_fluid_extrapolator.hpp, state/cuda/state_initialization.cuh,
material/cuda/combine_materials.cuh, simulator/multimaterial_simulator.hpp.
Bit-exactness: the ghost-fluid kernels are compiled without FMA contraction
and do their arithmetic in FP64 in the oracle's order, so the ghost pass
matches the oracle bit for bit in both state precisions.  The step loop adds
the split solver (FMA-contracted, 1e-12 per FP64 step) and the tile-ordered
reinitialisation, and is compared to 1e-7 (FP64) and 1e-4 (FP32) of each
component's largest magnitude.
"""
import numpy as np
import pytest

from fluidity_b200.workloads import shock_bubble


def _spec(seed=5, nx=128, ny=64):
    return shock_bubble(seed, nx=nx, ny=ny, width=2.0)


def _cons(prim, g):
    r, p, vx, vy = prim
    E = r * (0.5 * (vx * vx + vy * vy) + p / ((g - 1.0) * r))
    return np.array([r, E, r * vx, r * vy])


def _initial(spec, dtype=np.float64, perturb=0.0, seed=0):
    """Host copy of the shock-bubble initial data (as MultiMaterial.shock_bubble
    builds it on the device), optionally with a smooth perturbation."""
    from oracle import oracle as O
    n = spec["nx"] * spec["ny"]
    g0, g1 = spec["gammas"]
    u0 = np.zeros((4, n), dtype=dtype)
    u1 = np.zeros((4, n), dtype=dtype)
    allin = -np.ones(n)
    u0 = O.mm_set_states(u0, allin, spec["ambient"], g0)
    u0 = O.mm_set_states(u0, spec["shock_phi"], spec["shocked"], g0)
    u1 = O.mm_set_states(u1, allin, spec["bubble"], g1)
    if perturb:
        rng = np.random.default_rng(seed)
        nx, ny = spec["nx"], spec["ny"]
        X, Y = np.meshgrid(np.linspace(0, 1, nx), np.linspace(0, 1, ny))
        for u in (u0, u1):
            for c, scale in ((0, 0.1), (2, 0.2), (3, 0.2)):
                f = np.sin(2 * np.pi * (X * rng.integers(1, 4) + rng.uniform()))
                f *= np.cos(2 * np.pi * (Y * rng.integers(1, 4) + rng.uniform()))
                u[c] = (u[c] + perturb * scale * f.reshape(-1) * (1 if c else u[0])).astype(dtype)
    return u0, u1


def _relerr(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    # per component, floored at 1e-3 of the largest magnitude of any component
    scale = np.maximum(np.max(np.abs(b), axis=1, keepdims=True), 1e-3 * np.max(np.abs(b)))
    return float(np.max(np.abs(a - b) / scale))


# ---- oracle properties (CPU) --------------------------------------------------

def test_oracle_gfm_uniform_gas_is_fixed_point(oracle):
    """Same gas at rest on both sides: the star state is the state itself."""
    spec = _spec()
    n = spec["nx"] * spec["ny"]
    g = 1.4
    c = _cons([1.0, 1.0, 0.0, 0.0], g)
    u0 = np.tile(c[:, None], (1, n))
    u1 = u0.copy()
    a, b, written = oracle.mm_gfm(spec["nx"], spec["ny"], spec["h"], (g, g), u0, u1,
                                  spec["phi0"], spec["phi1"])
    assert written > 0
    assert _relerr(a, u0) < 1e-12 and _relerr(b, u1) < 1e-12


def test_oracle_extrapolation_keeps_constant_field(oracle):
    spec = _spec()
    n = spec["nx"] * spec["ny"]
    c = _cons([0.7, 2.0, 0.3, -0.2], 1.4)
    u = np.tile(c[:, None], (1, n))
    out, sweeps = oracle.mm_extrapolate(spec["nx"], spec["ny"], spec["h"], u, spec["phi1"])
    assert sweeps <= 2
    assert _relerr(out, u) < 1e-14


def test_oracle_extrapolation_fills_band_from_inside(oracle):
    """Material 1 (the bubble) holds gas A up to phi < dh (inside and the
    interface layer the GFM writes) and gas B beyond: the extrapolation pulls
    A into the band dh <= phi <= 6 dh/sqrt(2) along the normal (B leaks in
    only through the small tangential weights near the band's outer edge),
    and leaves every cell outside the band alone."""
    spec = _spec()
    h = spec["h"]
    inside = _cons([0.15, 1.0, 0.0, 0.0], 1.67)
    outside = _cons([1.0, 1.0, 0.0, 0.0], 1.67)
    phi = spec["phi1"]
    u = np.where(phi[None, :] < h, inside[:, None], outside[:, None])
    out, sweeps = oracle.mm_extrapolate(spec["nx"], spec["ny"], h, u, phi)
    assert 1 <= sweeps < 64
    band = (phi > 0) & (phi >= h) & (phi <= 6 * h / np.sqrt(2))
    assert band.sum() > 0
    frac = (out[0, band] - inside[0]) / (outside[0] - inside[0])
    assert np.median(frac) < 1e-6 and np.max(frac) < 0.25 and np.min(frac) >= -1e-12
    assert np.array_equal(out[:, ~band], u[:, ~band])


def test_oracle_set_states_and_combine(oracle):
    spec = _spec()
    n = spec["nx"] * spec["ny"]
    u = np.zeros((4, n))
    u = oracle.mm_set_states(u, spec["phi1"], spec["bubble"], 1.67)
    inside = spec["phi1"] <= 0
    assert np.allclose(u[:, inside], _cons(spec["bubble"], 1.67)[:, None], rtol=1e-15)
    assert np.all(u[:, ~inside] == 0)
    base = np.ones((4, n))
    merged = oracle.mm_combine(base, u, spec["phi1"])
    assert np.array_equal(merged[:, inside], u[:, inside])
    assert np.all(merged[:, ~inside] == 1)


def test_oracle_mm_step_runs(oracle):
    spec = _spec(nx=96, ny=48)
    u0, u1 = _initial(spec)
    p0, p1 = spec["phi0"], spec["phi1"]
    nx, ny, h = spec["nx"], spec["ny"], spec["h"]
    for k in range(3):
        u0, u1, p0, p1, dt = oracle.mm_step(nx, ny, h, spec["gammas"], 0.6, u0, u1, p0, p1,
                                            reinit=(k == 2))
        assert dt > 0 and np.isfinite(dt)
    assert np.all(np.isfinite(u0)) and np.all(np.isfinite(u1))
    assert np.array_equal(p0, -p1) or np.max(np.abs(p0 + p1)) < 1e-12 * np.max(np.abs(p0))


# ---- CUDA kernels vs the oracle -----------------------------------------------

def _device_mm(spec, dtype, u0, u1):
    import torch
    from fluidity_b200.multimaterial import MultiMaterial
    mm = MultiMaterial((spec["nx"], spec["ny"]), spec["gammas"], spec["h"], dtype=dtype)
    tdt = torch.float32 if dtype == "f32" else torch.float64
    mm.u[0][0].copy_(torch.as_tensor(u0, dtype=tdt))
    mm.u[1][0].copy_(torch.as_tensor(u1, dtype=tdt))
    mm.set_levelsets(spec["phi0"], spec["phi1"])
    return mm


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_set_states_combine_bit_exact(cuda, oracle, dtype):
    import torch
    from fluidity_b200.multimaterial import MultiMaterial
    spec = _spec(seed=9)
    npdt = np.float32 if dtype == "f32" else np.float64
    want0, want1 = _initial(spec, npdt)
    mm = MultiMaterial.shock_bubble(spec, dtype=dtype)
    got0, got1 = (t.cpu().numpy() for t in mm.states())
    assert np.array_equal(got0, want0) and np.array_equal(got1, want1)
    merged = mm.combine().cpu().numpy()
    assert np.array_equal(merged, oracle.mm_combine(want0, want1, spec["phi1"]))


@pytest.mark.gpu
@pytest.mark.parametrize("dtype,seed", [("f64", 1), ("f64", 2), ("f32", 3)])
def test_ghost_matches_oracle(cuda, oracle, dtype, seed):
    spec = _spec(seed=seed)
    npdt = np.float32 if dtype == "f32" else np.float64
    u0, u1 = _initial(spec, npdt, perturb=1.0, seed=seed)
    w0, w1 = oracle.mm_ghost(spec["nx"], spec["ny"], spec["h"], spec["gammas"], u0, u1,
                             spec["phi0"], spec["phi1"])
    mm = _device_mm(spec, dtype, u0, u1)
    mm.ghost()
    st = mm.stats()
    assert st["gfm0"] > 0 and st["gfm1"] > 0 and st["band0"] > 0 and st["band1"] > 0
    assert 1 <= st["extrap_iters0"] <= 64 and 1 <= st["extrap_iters1"] <= 64
    g0, g1 = (t.cpu().numpy() for t in mm.states())
    assert np.array_equal(g0, w0), _relerr(g0, w0)
    assert np.array_equal(g1, w1), _relerr(g1, w1)
    changed = np.any(w0 != u0, axis=0) | np.any(w1 != u1, axis=0)
    assert changed.sum() > 0


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_steps_match_oracle(cuda, oracle, dtype):
    spec = _spec(seed=4, nx=96, ny=48)
    npdt = np.float32 if dtype == "f32" else np.float64
    u0, u1 = _initial(spec, npdt)
    mm = _device_mm(spec, dtype, u0, u1)
    nsteps, every = 4, 2
    mm.begin(cfl=0.6, sim_time=1e9, max_iters=nsteps, reinit_every=every)
    mm.steps(nsteps)
    it, rt, done = mm.status()
    assert it == nsteps and done
    p0, p1 = spec["phi0"], spec["phi1"]
    t = 0.0
    for k in range(nsteps):
        u0, u1, p0, p1, dt = oracle.mm_step(spec["nx"], spec["ny"], spec["h"], spec["gammas"],
                                            0.6, u0, u1, p0, p1, reinit=((k + 1) % every == 0))
        t += dt
    assert abs(rt - t) < 1e-9 * t
    g0, g1 = (x.cpu().numpy() for x in mm.states())
    q0, q1 = (x.cpu().numpy() for x in mm.current_phi())
    tol = 1e-4 if dtype == "f32" else 1e-7
    assert _relerr(g0, u0) < tol, _relerr(g0, u0)
    assert _relerr(g1, u1) < tol, _relerr(g1, u1)
    assert np.max(np.abs(q0 - p0)) < tol * np.max(np.abs(p0))
    assert np.max(np.abs(q1 - p1)) < tol * np.max(np.abs(p1))


def test_mm_rejects_bad_arguments():
    import ctypes as C
    from fluidity_b200 import capi
    lib = capi.load()
    h = C.c_void_p()
    g = capi.Grid.make((64,))
    gam = (C.c_double * 2)(1.4, 1.67)
    assert lib.fl_mm_create(C.byref(h), C.byref(g), gam, 0, 0.01) == capi.FL_EINVAL
    g = capi.Grid.make((64, 64))
    bad = (C.c_double * 2)(1.0, 1.67)
    assert lib.fl_mm_create(C.byref(h), C.byref(g), bad, 0, 0.01) == capi.FL_EINVAL
    assert lib.fl_mm_steps(None, 1, None) == capi.FL_EINVAL
