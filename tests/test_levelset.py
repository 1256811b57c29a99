"""Level-set operations of the multimaterial path: the oracle's properties on
CPU, then the CUDA kernels against the oracle on the same seeded inputs.

Reference: levelset/cuda/velocity_initialization.cuh, scheme/cuda/evolve.cuh
with scheme/updaters/runge_kutta_3.hpp and scheme/stencils/weno_hj_5.hpp,
levelset/cuda/levelset_projection.cuh, scheme/cuda/fast_iterative_method.cuh.
Bit-exactness: the velocity and projection kernels are compiled without FMA
contraction and use IEEE division and square root, so they match the oracle
bit for bit.  The RK3 advection contracts into FMAs and normalises the WENO
weights with one reciprocal per derivative; it agrees with the oracle to
1e-12 of max |phi|, one step or twenty.  The reinitialisation relaxes in a
different order (16x16 tiles against whole-grid Jacobi sweeps); its fixed
point agrees to 1e-12 of max |phi|.
"""
import numpy as np
import pytest


def circle_phi(nx, ny, seed, wobble=0.3):
    """A perturbed circle level set (not a distance function): negative inside."""
    rng = np.random.default_rng(seed)
    cx, cy = rng.uniform(0.4, 0.6, 2)
    r0 = rng.uniform(0.2, 0.3)
    h = 1.0 / nx
    x = (np.arange(nx) + 0.5) * h
    y = (np.arange(ny) + 0.5) * h
    X, Y = np.meshgrid(x, y)
    r = np.hypot(X - cx, Y - cy)
    th = np.arctan2(Y - cy, X - cx)
    phi = (r - r0) * (1.0 + wobble * np.sin(3 * th))
    return phi.reshape(-1), h


def gas_state(nx, ny, seed, pitch=None):
    """SoA (rho, E, m_x, m_y) planes with smooth velocities."""
    rng = np.random.default_rng(seed)
    n = nx * ny
    pitch = n if pitch is None else pitch
    x = np.linspace(0, 1, nx, endpoint=False)
    y = np.linspace(0, 1, ny, endpoint=False)
    X, Y = np.meshgrid(x, y)
    rho = 1.0 + 0.5 * np.sin(2 * np.pi * (X + rng.uniform()))
    u = np.cos(2 * np.pi * (Y + rng.uniform()))
    v = 0.5 * np.sin(2 * np.pi * (X + Y + rng.uniform()))
    p = 1.0 + 0.2 * np.cos(2 * np.pi * X)
    st = np.zeros((4, pitch))
    st[0, :n] = rho.reshape(-1)
    st[2, :n] = (rho * u).reshape(-1)
    st[3, :n] = (rho * v).reshape(-1)
    st[1, :n] = (p / 0.4 + 0.5 * rho * (u * u + v * v)).reshape(-1)
    return st


# ---- oracle properties (CPU) --------------------------------------------------

def test_oracle_reinit_plane_is_exact(oracle):
    """phi = 3 (x - x0): the one source is the cell nearest x0 (it keeps
    |phi|); every other cell sits a whole number of cells further away."""
    nx, ny = 40, 24
    h = 1.0 / nx
    x0 = 0.4321
    x = (np.arange(nx) + 0.5) * h
    phi = np.tile(3.0 * (x - x0), ny)           # slope 3: not a distance
    d, sweeps = oracle.ls_reinit(nx, ny, phi, h)
    assert 0 < sweeps < 200
    near = int(np.argmin(np.abs(x - x0)))
    want = np.sign(x - x0) * (3.0 * abs(x[near] - x0) + np.abs(np.arange(nx) - near) * h)
    assert np.max(np.abs(d - np.tile(want, ny))) < 1e-12


def test_oracle_reinit_circle_is_distance(oracle):
    nx = ny = 64
    phi, h = circle_phi(nx, ny, 5, wobble=0.0)   # exact distance to a circle
    d, _ = oracle.ls_reinit(nx, ny, phi, h)
    # first-order Godunov distance: within a cell of the exact distance
    exact = phi
    assert np.max(np.abs(d - exact)) < 1.0 * h
    g = np.gradient(d.reshape(ny, nx), h)
    mag = np.hypot(*g)
    band = (np.abs(exact.reshape(ny, nx)) > 3 * h) & (np.abs(exact.reshape(ny, nx)) < 0.15)
    assert np.median(np.abs(mag[band] - 1.0)) < 0.05


def test_oracle_advect_linear_exact(oracle):
    nx, ny = 48, 16
    h = 1.0 / nx
    x = (np.arange(nx) + 0.5) * h
    phi = np.tile(x - 0.5, ny)
    vel = np.full(nx * ny, 0.75)
    dt = 0.3 * h
    out = oracle.ls_advect(nx, ny, phi, vel, dt, h)
    # |grad phi| = 1 beyond the three stages' reach (3 x 3 cells) of the
    # mirrored ends: there phi decreases by v dt
    inner = np.tile((np.arange(nx) >= 9) & (np.arange(nx) < nx - 9), ny)
    assert np.max(np.abs(out[inner] - (phi[inner] - 0.75 * dt))) < 1e-13


def test_oracle_project(oracle):
    rng = np.random.default_rng(4)
    a = rng.normal(size=1000)
    b = rng.normal(size=1000)
    pa, pb = oracle.ls_project(a, b)
    assert np.array_equal(pa, -pb)
    assert np.allclose(pa, (a - b) / 2, rtol=0, atol=1e-15)


def test_oracle_velocity_uniform(oracle):
    nx, ny = 20, 12
    h = 1.0 / nx
    x = (np.arange(nx) + 0.5) * h
    phi = np.tile(x - 0.5, ny)
    st = gas_state(nx, ny, 0)
    st[2] = st[0] * 1.5                            # u = 1.5, v = 0
    st[3] = 0.0
    v = oracle.ls_velocity(nx, ny, [phi], [st], h)
    inside = phi <= 0
    assert np.allclose(v[inside], 1.5, rtol=0, atol=1e-14)
    assert np.all(v[~inside] == 0.0)


# ---- CUDA kernels vs the oracle -----------------------------------------------

# The advection's bar against the oracle: max |got - want| over max |want|.
ADVECT_TOL = 1e-12


def _maxrel(got, want):
    return float(np.max(np.abs(got - want)) / np.max(np.abs(want)))


def _ops(shape):
    from fluidity_b200.levelset import LevelSetOps
    return LevelSetOps(shape)


@pytest.mark.gpu
@pytest.mark.parametrize("nx,ny,seed", [(64, 48, 1), (33, 70, 2), (200, 130, 3)])
def test_advect_matches_oracle(cuda, oracle, nx, ny, seed):
    import torch
    phi, h = circle_phi(nx, ny, seed)
    vel = oracle.ls_velocity(nx, ny, [phi], [gas_state(nx, ny, seed)], h)
    dt = 0.4 * h
    want = oracle.ls_advect(nx, ny, phi, vel, dt, h)
    ops = _ops((nx, ny))
    got = ops.advect(torch.tensor(phi, device=cuda), torch.tensor(vel, device=cuda), dt, h)
    # the RK3 stages contract products into FMAs and normalise the WENO
    # weights with one reciprocal: rounding-level agreement
    assert _maxrel(got.cpu().numpy(), want) <= ADVECT_TOL


@pytest.mark.gpu
def test_advect_many_steps(cuda, oracle):
    import torch
    nx, ny = 96, 80
    phi, h = circle_phi(nx, ny, 7)
    vel = np.full(nx * ny, -0.8)
    dt = 0.5 * h
    ops = _ops((nx, ny))
    a = torch.tensor(phi, device=cuda)
    b = ops.new()
    v = torch.tensor(vel, device=cuda)
    want = phi
    for _ in range(20):
        want = oracle.ls_advect(nx, ny, want, vel, dt, h)
        ops.advect(a, v, dt, h, out=b)
        a, b = b, a
    assert _maxrel(a.cpu().numpy(), want) <= ADVECT_TOL


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_velocity_matches_oracle(cuda, oracle, dtype):
    import torch
    nx, ny = 70, 45
    phi0, h = circle_phi(nx, ny, 11)
    phi1 = -phi0 + 0.01
    pitch = nx * ny + 13
    s0 = gas_state(nx, ny, 11, pitch)
    s1 = gas_state(nx, ny, 12, pitch)
    tdt = torch.float64 if dtype == "f64" else torch.float32
    if dtype == "f32":   # the oracle sees the same rounded states
        s0 = s0.astype(np.float32).astype(np.float64)
        s1 = s1.astype(np.float32).astype(np.float64)
    want = oracle.ls_velocity(nx, ny, [phi0, phi1], [s0, s1], h)
    ops = _ops((nx, ny))
    p = [torch.tensor(phi0, device=cuda), torch.tensor(phi1, device=cuda)]
    s = [torch.tensor(s0, device=cuda, dtype=tdt), torch.tensor(s1, device=cuda, dtype=tdt)]
    got = ops.velocity(p, s, h, dtype=dtype).cpu().numpy()
    assert np.array_equal(got, want)


@pytest.mark.gpu
def test_project_bit_exact(cuda, oracle):
    import torch
    rng = np.random.default_rng(9)
    a = rng.normal(size=12345)
    b = rng.normal(size=12345)
    wa, wb = oracle.ls_project(a, b)
    ta = torch.tensor(a, device=cuda)
    tb = torch.tensor(b, device=cuda)
    _ops((111, 111)).project(ta, tb)
    assert np.array_equal(ta.cpu().numpy(), wa)
    assert np.array_equal(tb.cpu().numpy(), wb)


@pytest.mark.gpu
@pytest.mark.parametrize("nx,ny,seed,scale", [(64, 64, 1, 2.5), (100, 37, 2, 0.7),
                                              (257, 129, 3, 1.0)])
def test_reinit_matches_oracle(cuda, oracle, nx, ny, seed, scale):
    import torch
    phi, h = circle_phi(nx, ny, seed)
    phi = phi * scale
    want, sweeps = oracle.ls_reinit(nx, ny, phi, h)
    ops = _ops((nx, ny))
    got = ops.reinit(torch.tensor(phi, device=cuda), h).cpu().numpy()
    assert 0 < ops.passes < 10 * (nx + ny)
    assert np.array_equal(np.sign(got), np.sign(phi))
    err = np.max(np.abs(got - want))
    assert err < 1e-12 * np.max(np.abs(want)), (err, sweeps, ops.passes)


@pytest.mark.gpu
def test_reinit_is_deterministic_and_odd(cuda):
    """Repeated calls give identical results, and reinit(-phi) = -reinit(phi)
    bit for bit (the two-material path relies on it: its level sets are
    reinitialised separately and must stay negatives of each other)."""
    import torch
    nx, ny = 300, 170
    phi, h = circle_phi(nx, ny, 6)
    phi = phi * 1.3
    ops = _ops((nx, ny))
    t = torch.tensor(phi, device=cuda)
    a = ops.reinit(t, h).cpu().numpy()
    for _ in range(3):
        assert np.array_equal(ops.reinit(t, h).cpu().numpy(), a)
    b = ops.reinit(-t, h).cpu().numpy()
    assert np.array_equal(b, -a)


@pytest.mark.gpu
def test_reinit_pass_limit_reports_timeout(cuda):
    import torch
    from fluidity_b200 import capi
    nx, ny = 128, 128
    phi, h = circle_phi(nx, ny, 4)
    ops = _ops((nx, ny))
    with pytest.raises(capi.FlError) as e:
        ops.reinit(torch.tensor(phi, device=cuda), h, max_passes=1)
    assert e.value.code == capi.FL_ETIMEOUT
    assert ops.passes == 1


def test_levelset_rejects_bad_grids():
    from fluidity_b200 import capi
    lib = capi.load()
    g = capi.Grid.make((64,))
    assert lib.fl_ls_workspace_bytes(C_ref(g)) == -1
    g = capi.Grid.make((3, 64))
    assert lib.fl_ls_workspace_bytes(C_ref(g)) == -1
    g = capi.Grid.make((64, 64))
    assert lib.fl_ls_workspace_bytes(C_ref(g)) >= 2 * 64 * 64 * 8 + 64 * 64


def C_ref(g):
    import ctypes
    return ctypes.byref(g)
