"""The discrete adjoint on the GPU: single sweeps against finite differences
of the forward sweep, the checkpointed time loop against central finite
differences of the objective J = 0.5 ||p(T) - p_target||^2 along seeded
directions (time steps frozen), and checkpoint-interval independence."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GAMMA = 1.4


def _smooth_state(shape, seed, narrow_p=False):
    from _util import random_prim
    from oracle import oracle
    prim = random_prim(shape, seed, smooth=True, mild=True)
    if narrow_p:
        # pressure within 1 +- 5 %: the flattening test |dp| / p > 0.33 never
        # passes, so chi = 1 and freezing it is exact
        prim[1] = 1.0 + 0.1 * (prim[1] - prim[1].min()) / (np.ptp(prim[1]) + 1e-30) - 0.05
    return oracle.prim_to_cons(prim, GAMMA)


@pytest.mark.parametrize("shape,dim", [((64,), 0), ((40, 24), 0), ((40, 24), 1)])
@pytest.mark.parametrize("flux", ["hllc", "force"])
@pytest.mark.parametrize("reflect", [0, 1])
@pytest.mark.parametrize("flatten", [False, True])
def test_adjoint_sweep_transpose(cuda, shape, dim, flux, reflect, flatten):
    """<lam, J du> (central differences of fl_split_sweep) = <J^T lam, du>.
    The adjoint freezes the flattening coefficient chi, so the check runs
    without flattening, and with flattening on data where it stays inactive."""
    import torch
    from fluidity_b200 import capi
    from fluidity_b200.solver import SplitSolver
    lib = capi.load()
    u = torch.from_numpy(_smooth_state(shape, 3 + dim, narrow_p=flatten)).cuda()
    s = SplitSolver(shape, flux=flux, gamma=GAMMA, boundary_mask=reflect, flatten=flatten)
    ws = s.max_wavespeed(u).item()
    dtdh = 0.6 / ws
    g = torch.Generator(device="cpu").manual_seed(11)
    lam = torch.randn(u.shape, generator=g, dtype=torch.float64).cuda()
    du = (torch.randn(u.shape, generator=g, dtype=torch.float64) * 1e-2).cuda() * u.abs()
    eps = 1e-6
    up, um = torch.empty_like(u), torch.empty_like(u)
    s.sweep(u + eps * du, up, dim, dtdh)
    s.sweep(u - eps * du, um, dim, dtdh)
    fd = torch.sum(lam * (up - um)).item() / (2 * eps)
    lam_in = torch.empty_like(u)
    capi.check(lib.fl_adjoint_sweep(C.byref(s.grid), dim, C.c_void_p(u.data_ptr()),
                                    C.c_void_p(lam.data_ptr()), C.c_void_p(lam_in.data_ptr()),
                                    GAMMA, dtdh, s.policy, reflect, None))
    torch.cuda.synchronize()
    ad = torch.sum(lam_in * du).item()
    assert abs(fd - ad) <= 1e-6 * max(abs(ad), 1e-12), (fd, ad)


@pytest.mark.parametrize("seed", [5, 6, 9, 11])
@pytest.mark.parametrize("dim", [0, 1])
@pytest.mark.parametrize("flux", ["hllc", "force"])
def test_adjoint_sweep_reflective_walls(cuda, seed, dim, flux):
    """Reflective walls at both ends of the sweep: the ghost cells' adjoints
    fold back onto the cells they mirror, including the part through the
    wall cell's own slope (non-zero where the limiter takes the normal
    momentum's difference across the wall, 2 m).  Seeds 6 and 9 put a
    normal velocity near zero at a wall."""
    import torch
    from fluidity_b200 import capi
    from fluidity_b200.solver import SplitSolver
    lib = capi.load()
    shape = (40, 24)
    u = torch.from_numpy(_smooth_state(shape, seed)).cuda()
    reflect = 1 << dim
    s = SplitSolver(shape, flux=flux, gamma=GAMMA, boundary_mask=reflect, flatten=False)
    dtdh = 0.6 / s.max_wavespeed(u).item()
    g = torch.Generator(device="cpu").manual_seed(13)
    lam = torch.randn(u.shape, generator=g, dtype=torch.float64).cuda()
    du = (torch.randn(u.shape, generator=g, dtype=torch.float64) * 1e-2).cuda() * u.abs()
    eps = 1e-6
    up, um = torch.empty_like(u), torch.empty_like(u)
    s.sweep(u + eps * du, up, dim, dtdh)
    s.sweep(u - eps * du, um, dim, dtdh)
    fd = torch.sum(lam * (up - um)).item() / (2 * eps)
    lam_in = torch.empty_like(u)
    capi.check(lib.fl_adjoint_sweep(C.byref(s.grid), dim, C.c_void_p(u.data_ptr()),
                                    C.c_void_p(lam.data_ptr()), C.c_void_p(lam_in.data_ptr()),
                                    GAMMA, dtdh, s.policy, reflect, None))
    torch.cuda.synchronize()
    ad = torch.sum(lam_in * du).item()
    assert abs(fd - ad) <= 1e-6 * max(abs(ad), 1e-12), (fd, ad)


def _smooth_density(n, seed):
    """1 + a few low Fourier modes: smooth everywhere, no flat regions."""
    import torch
    g = torch.Generator(device="cpu").manual_seed(seed)
    x = (torch.arange(n, dtype=torch.float64) + 0.5) / n
    X, Y = x.repeat(n), x.repeat_interleave(n)
    rho = torch.ones(n * n, dtype=torch.float64)
    for kx, ky in ((1, 1), (2, 1), (1, 3)):
        a, px, py = torch.rand(3, generator=g, dtype=torch.float64) * torch.tensor([0.3, 6.3, 6.3])
        rho = rho + a * torch.sin(2 * torch.pi * kx * X + px) * torch.sin(2 * torch.pi * ky * Y + py)
    return rho.cuda()


def _gradient_case(shape, nsteps, interval, seed=1, flatten=True, recon="muscl", count=8,
                   smooth=False):
    import torch
    from fluidity_b200.adjoint import (Adjoint, gaussian_density, objective, pressure, rollout,
                                       state_from_density)
    n = shape[0]
    if smooth:
        rho0 = _smooth_density(n, seed).requires_grad_(True)
        target = _smooth_density(n, seed + 100)
    else:
        rho0 = gaussian_density(n, seed, count=count).requires_grad_(True)
        target = gaussian_density(n, seed + 100, count=count)
    adj = Adjoint(shape, nsteps, interval=interval, flatten=flatten, recon=recon)
    with torch.no_grad():
        p_target = pressure(adj.forward(state_from_density(target), 0.7))
    u0 = state_from_density(rho0)
    uN = rollout(u0, adj, 0.7)
    J = objective(uN, p_target)
    J.backward()
    return rho0, adj, p_target, J.item(), rho0.grad.clone()


def _fd_errors(rho0, adj, p_target, grad, count, eps=1e-6):
    import math
    import torch
    from fluidity_b200.adjoint import objective_difference, random_directions, state_from_density
    dts = adj.dtdh()
    errs = []
    for v in random_directions(rho0.numel(), count, seed=7):
        with torch.no_grad():
            up = adj.forward(state_from_density(rho0 + eps * v), 0.7, frozen_dtdh=dts)
            um = adj.forward(state_from_density(rho0 - eps * v), 0.7, frozen_dtdh=dts)
        fd = objective_difference(up, um, p_target).item() / (2 * eps)
        ad = torch.dot(grad, v).item()
        r = abs(fd - ad) / max(abs(ad), 1e-30)
        assert math.isfinite(r), (fd, ad)
        errs.append(r)
    return errs


# The discrete step is piecewise smooth: the minmod limiter switches where
# the one-sided differences cross, HLLC's wave-speed estimate switches between
# its shock and rarefaction forms.  A central difference whose +-eps interval
# straddles a switch averages two one-sided derivatives; such straddles are
# common where a field is flat to round-off (Gaussian tails), because every
# limiter there decides on differences far below eps.  The MUSCL checks
# therefore run on smooth Fourier-mode densities.

def test_adjoint_gradient_first_order_matches_finite_differences(cuda):
    """Piecewise-constant reconstruction (no limiter): every direction agrees
    with central differences to 1e-6."""
    import torch
    rho0, adj, p_target, J0, grad = _gradient_case((48, 48), nsteps=24, interval=5,
                                                   recon="basic", count=32)
    assert J0 > 0 and torch.norm(grad).item() > 0
    errs = _fd_errors(rho0.detach(), adj, p_target, grad, 6)
    print("first order, adjoint vs central differences:", ["%.2e" % e for e in errs])
    assert max(errs) < 1e-6


def test_adjoint_gradient_muscl_matches_finite_differences(cuda):
    """MUSCL-Hancock without flattening on smooth data: half the directions
    agree to 1e-6 and the median to 1e-5; the others straddle a limiter
    switch inside +-eps (a systematic error would move every direction)."""
    import statistics
    import torch
    rho0, adj, p_target, J0, grad = _gradient_case((48, 48), nsteps=8, interval=3,
                                                   flatten=False, smooth=True)
    assert J0 > 0 and torch.norm(grad).item() > 0
    errs = _fd_errors(rho0.detach(), adj, p_target, grad, 8)
    print("MUSCL, adjoint vs central differences:", ["%.2e" % e for e in errs])
    # about one limiter switch per direction falls inside +-eps at this size
    assert statistics.median(errs) < 1e-5
    assert sum(e < 1e-6 for e in errs) >= 4
    assert max(errs) < 1e-3


def test_adjoint_gradient_with_flattening(cuda):
    """With flattening on (chi differentiated through its ramp), against
    central differences on a smooth field: reported, and held to the FD
    noise and limiter-switch level of this field."""
    import torch
    rho0, adj, p_target, J0, grad = _gradient_case((48, 48), nsteps=8, interval=3, smooth=True)
    assert J0 > 0 and torch.norm(grad).item() > 0
    errs = _fd_errors(rho0.detach(), adj, p_target, grad, 4)
    print("MUSCL + flattening, adjoint vs central differences:", ["%.2e" % e for e in errs])
    assert max(errs) < 5e-2


@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_adjoint_driver_equals_sweep_composition(cuda, dtype):
    """The checkpointed reverse pass (fl_adj_backward) is exactly the
    composition of single-sweep adjoints (fl_adjoint_sweep) taken at the
    forward pass's sweep inputs, in reverse order, with the recorded time
    steps -- so the FD agreement of single sweeps carries over to the whole
    rollout."""
    import torch
    from fluidity_b200 import capi
    from fluidity_b200.adjoint import Adjoint, gaussian_density, state_from_density
    from fluidity_b200.solver import SplitSolver
    lib = capi.load()
    n, nsteps = 48, 5
    tdt = torch.float64 if dtype == "f64" else torch.float32
    u0 = state_from_density(gaussian_density(n, 3, count=32, dtype=tdt)).contiguous()
    adj = Adjoint((n, n), nsteps, dtype=dtype, interval=2)
    adj.forward(u0, 0.7)
    dts = adj.dtdh()
    s = SplitSolver((n, n), dtype=dtype)
    inputs = []
    cur = u0.clone()
    for k in range(nsteps):
        for d in range(2):
            nxt = torch.empty_like(cur)
            inputs.append((k, d, cur))
            s.sweep(cur, nxt, d, float(dts[k]))
            cur = nxt
    g = torch.Generator(device="cpu").manual_seed(4)
    lam = torch.randn(u0.shape, generator=g, dtype=torch.float64).to(device=u0.device, dtype=tdt)
    want = lam.clone()
    for k, d, uin in reversed(inputs):
        out = torch.empty_like(want)
        capi.check(lib.fl_adjoint_sweep(C.byref(s.grid), d, C.c_void_p(uin.data_ptr()),
                                        C.c_void_p(want.data_ptr()), C.c_void_p(out.data_ptr()),
                                        GAMMA, float(dts[k]), s.policy, 0, None))
        want = out
    got = adj.backward(lam)
    torch.cuda.synchronize()
    assert torch.equal(got, want)


def test_adjoint_checkpoint_interval_independent(cuda):
    import torch
    _, _, _, J1, g1 = _gradient_case((32, 32), nsteps=13, interval=1)
    _, _, _, J2, g2 = _gradient_case((32, 32), nsteps=13, interval=4)
    _, _, _, J3, g3 = _gradient_case((32, 32), nsteps=13, interval=0)
    assert J1 == J2 == J3
    assert torch.equal(g1, g2) and torch.equal(g1, g3)


def test_adjoint_1d(cuda):
    """1-D tube: the rollout's gradient against central differences."""
    import torch
    from fluidity_b200.adjoint import Adjoint
    shape = (128,)
    u0 = torch.from_numpy(_smooth_state(shape, 21)).cuda()
    adj = Adjoint(shape, 30, interval=6)
    uN = adj.forward(u0, 0.8)
    dts = adj.dtdh()
    g = torch.Generator(device="cpu").manual_seed(5)
    lamN = torch.randn(uN.shape, generator=g, dtype=torch.float64).cuda()
    lam0 = adj.backward(lamN)
    du = (torch.randn(u0.shape, generator=g, dtype=torch.float64) * 1e-2).cuda() * u0.abs()
    eps = 1e-6
    up = adj.forward(u0 + eps * du, 0.8, frozen_dtdh=dts)
    um = adj.forward(u0 - eps * du, 0.8, frozen_dtdh=dts)
    fd = torch.sum(lamN * (up - um)).item() / (2 * eps)
    ad = torch.sum(lam0 * du).item()
    assert abs(fd - ad) <= 1e-6 * abs(ad), (fd, ad)


# ---- the stiffened fluid (p + p_inf under the sound speed) -------------------

P_INF = 2.0


@pytest.mark.parametrize("shape,dim", [((64,), 0), ((40, 24), 0), ((40, 24), 1)])
@pytest.mark.parametrize("flux", ["hllc", "force"])
@pytest.mark.parametrize("reflect", [0, 1])
def test_adjoint_sweep_transpose_stiff(cuda, shape, dim, flux, reflect):
    """fl_adjoint_sweep_mat against central differences of the stiffened
    fluid's forward sweep (fl_split_sweep_mat), flattening off."""
    import torch
    from fluidity_b200 import capi
    from fluidity_b200.solver import SplitSolver
    lib = capi.load()
    u = torch.from_numpy(_smooth_state(shape, 5 + dim)).cuda()
    s = SplitSolver(shape, flux=flux, gamma=GAMMA, boundary_mask=reflect, flatten=False,
                    p_inf=P_INF)
    ws = s.max_wavespeed(u).item()
    dtdh = 0.6 / ws
    g = torch.Generator(device="cpu").manual_seed(13)
    lam = torch.randn(u.shape, generator=g, dtype=torch.float64).cuda()
    du = (torch.randn(u.shape, generator=g, dtype=torch.float64) * 1e-2).cuda() * u.abs()
    eps = 1e-6
    up, um = torch.empty_like(u), torch.empty_like(u)
    s.sweep(u + eps * du, up, dim, dtdh)
    s.sweep(u - eps * du, um, dim, dtdh)
    fd = torch.sum(lam * (up - um)).item() / (2 * eps)
    lam_in = torch.empty_like(u)
    mat = capi.Material(GAMMA, P_INF)
    capi.check(lib.fl_adjoint_sweep_mat(C.byref(s.grid), dim, C.c_void_p(u.data_ptr()),
                                        C.c_void_p(lam.data_ptr()),
                                        C.c_void_p(lam_in.data_ptr()), C.byref(mat), dtdh,
                                        s.policy, reflect, None))
    torch.cuda.synchronize()
    ad = torch.sum(lam_in * du).item()
    assert abs(fd - ad) <= 1e-6 * max(abs(ad), 1e-12), (fd, ad)
    if flux == "hllc":
        # the ideal-gas adjoint is a different transpose: p_inf reaches it
        lam_ig = torch.empty_like(u)
        capi.check(lib.fl_adjoint_sweep(C.byref(s.grid), dim, C.c_void_p(u.data_ptr()),
                                        C.c_void_p(lam.data_ptr()),
                                        C.c_void_p(lam_ig.data_ptr()), GAMMA, dtdh, s.policy,
                                        reflect, None))
        torch.cuda.synchronize()
        assert not torch.equal(lam_ig, lam_in)


def test_adjoint_stiff_rollout(cuda):
    """Checkpointed rollout of the stiffened fluid: the recorded first step is
    the stiff CFL step, the forward pass equals fl_split_sweep_mat applied
    with the recorded steps, and the gradient matches central differences."""
    import torch
    from fluidity_b200.adjoint import Adjoint
    from fluidity_b200.solver import SplitSolver
    shape = (128,)
    u0 = torch.from_numpy(_smooth_state(shape, 23)).cuda()
    adj = Adjoint(shape, 30, interval=6, flatten=False, p_inf=P_INF)
    uN = adj.forward(u0, 0.8)
    dts = adj.dtdh()
    s = SplitSolver(shape, gamma=GAMMA, flatten=False, p_inf=P_INF)
    ws = s.max_wavespeed(u0).item()
    assert dts[0] == pytest.approx(0.8 / ws, rel=1e-14)
    ws_ideal = SplitSolver(shape, gamma=GAMMA, flatten=False).max_wavespeed(u0).item()
    assert ws > ws_ideal
    cur = u0.clone()
    for k in range(30):
        nxt = torch.empty_like(cur)
        s.sweep(cur, nxt, 0, float(dts[k]))
        cur = nxt
    torch.cuda.synchronize()
    assert torch.equal(cur, uN)
    g = torch.Generator(device="cpu").manual_seed(6)
    lamN = torch.randn(uN.shape, generator=g, dtype=torch.float64).cuda()
    lam0 = adj.backward(lamN)
    du = (torch.randn(u0.shape, generator=g, dtype=torch.float64) * 1e-2).cuda() * u0.abs()
    eps = 1e-6
    up = adj.forward(u0 + eps * du, 0.8, frozen_dtdh=dts)
    um = adj.forward(u0 - eps * du, 0.8, frozen_dtdh=dts)
    fd = torch.sum(lamN * (up - um)).item() / (2 * eps)
    ad = torch.sum(lam0 * du).item()
    assert abs(fd - ad) <= 1e-6 * abs(ad), (fd, ad)


def test_adjoint_set_material_drops_the_forward_pass(cuda):
    import torch
    from fluidity_b200 import capi
    from fluidity_b200.adjoint import Adjoint
    shape = (64,)
    u0 = torch.from_numpy(_smooth_state(shape, 29)).cuda()
    adj = Adjoint(shape, 4)
    uN = adj.forward(u0, 0.8)
    mat = capi.Material(GAMMA, P_INF)
    capi.check(adj.lib.fl_adj_set_material(adj.handle, C.byref(mat)), adj.lib)
    with pytest.raises(capi.FlError):
        adj.backward(torch.ones_like(uN))
    bad = capi.Material(GAMMA, -1.0)
    assert adj.lib.fl_adj_set_material(adj.handle, C.byref(bad)) != 0


def _dual_directional(rho0, dts, p_target, v, gamma=1.4, chi_diff=True, **pol):
    """J'(rho0)[v] from the oracle's sweep in forward-mode dual numbers
    (oracle/fl_oracle_dual.cpp) over the frozen time steps: the exact
    derivative of the discrete map whose branches and dt are those of the
    forward pass, with the flattening coefficient differentiated through its
    ramp (chi_diff; frozen otherwise) -- the map the adjoint transposes."""
    import numpy as np
    from oracle import oracle
    n = int(round(rho0.size ** 0.5))
    shape = (n, n)
    z = np.zeros_like(rho0)
    u0 = np.stack([rho0, rho0 / (gamma - 1.0), z, z])     # state_from_density, p = rho
    du0 = np.stack([v, v / (gamma - 1.0), z, z])
    u, du = oracle.rollout_dual(shape, u0, du0, gamma, dts, chi_diff=chi_diff, **pol)
    rho, e, mx, my = u
    drho, de, dmx, dmy = du
    ke = 0.5 * (mx * mx + my * my) / rho
    dke = (mx * dmx + my * dmy) / rho - ke * drho / rho
    p = (gamma - 1.0) * (e - ke)
    dp = (gamma - 1.0) * (de - dke)
    return float(np.sum((p - p_target) * dp))


def _ramp_case(n=48, nsteps=8, interval=3):
    """A density ramp from 1 to 4 over two cells along a tilted line, at rest
    with p = rho: the pressure jump launches a shock whose compression turns
    the flattening coefficient on (chi < 1) from the second step."""
    import torch
    from fluidity_b200.adjoint import Adjoint, objective, pressure, rollout, state_from_density
    x = (torch.arange(n, dtype=torch.float64) + 0.5) / n
    X, Y = x.repeat(n), x.repeat_interleave(n)
    rho0 = (1.0 + 3.0 * torch.clamp((X + 0.3 * Y - 0.55) * n / 2.0, 0.0, 1.0)).cuda()
    target = (1.0 + 0.2 * torch.sin(2 * torch.pi * X) * torch.cos(2 * torch.pi * Y)).cuda()
    rho0.requires_grad_(True)
    adj = Adjoint((n, n), nsteps, interval=interval, flatten=True)
    with torch.no_grad():
        p_target = pressure(adj.forward(state_from_density(target), 0.7))
    J = objective(rollout(state_from_density(rho0), adj, 0.7), p_target)
    J.backward()
    return rho0, adj, p_target, J.item(), rho0.grad.clone()


@pytest.mark.parametrize("case", ["smooth", "smooth_flatten_on", "ramp_flatten_active"])
def test_adjoint_gradient_matches_fp64_reference_gradient(cuda, oracle, case):
    """The adjoint's gradient against an independent FP64 reference gradient:
    directional derivatives along seeded directions computed in forward-mode
    dual numbers through the CPU oracle's own sweep, with the forward pass's
    time steps and the flattening coefficient differentiated through its
    ramp.  Both are exact derivatives of the same frozen-branch map, so they
    agree to rounding: 1e-12 relative per direction, where finite
    differences stop at their noise floor and at every limiter switch inside
    +-eps.  The ramp case has the flattening coefficient active and on its
    ramp: the oracle's rollouts with and without flattening differ, and the
    derivative with chi frozen differs from the one with chi differentiated,
    so the chi terms are part of what is checked."""
    import numpy as np
    import torch
    from fluidity_b200.adjoint import random_directions
    flatten = case != "smooth"
    if case == "ramp_flatten_active":
        rho0, adj, p_target, J0, grad = _ramp_case()
    else:
        rho0, adj, p_target, J0, grad = _gradient_case((48, 48), nsteps=8, interval=3,
                                                       flatten=flatten, smooth=True)
    dts = adj.dtdh()
    if case == "ramp_flatten_active":
        r = rho0.detach().cpu().numpy()
        z = np.zeros_like(r)
        u0 = np.stack([r, r / 0.4, z, z])
        on, _ = oracle.rollout_dual((48, 48), u0, z.repeat(4).reshape(4, -1), 1.4, dts)
        off, _ = oracle.rollout_dual((48, 48), u0, z.repeat(4).reshape(4, -1), 1.4, dts,
                                     flatten=False)
        assert not np.array_equal(on, off), "flattening never triggered"
    r0 = rho0.detach().cpu().numpy()
    pt = p_target.cpu().numpy()
    errs = []
    chi_terms = []
    for v in random_directions(r0.size, 4, seed=11):
        ref = _dual_directional(r0, dts, pt, v.cpu().numpy(), flatten=flatten)
        ad = torch.dot(grad, v).item()
        errs.append(abs(ad - ref) / abs(ref))
        frozen = _dual_directional(r0, dts, pt, v.cpu().numpy(), chi_diff=False, flatten=flatten)
        chi_terms.append(abs(frozen - ref) / abs(ref))
    print("adjoint vs dual-number reference gradient:", ["%.2e" % e for e in errs],
          "; chi terms:", ["%.2e" % e for e in chi_terms])
    assert max(errs) < 1e-12
    if case == "ramp_flatten_active":
        assert max(chi_terms) > 1e-6, "chi never on its ramp"
