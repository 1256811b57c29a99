"""Discrete adjoint of the split-solver time loop (fl_adj_* in
include/fluidity_b200.h) and a thin torch.autograd.Function around it.

The rollout u0 -> u_N (nsteps of dimensionally split MUSCL-Hancock with the
CFL time step recorded on the forward pass and then frozen) is one autograd
node: its backward runs the hand-written adjoint with sqrt(N) checkpointing.
Objectives and the parametrisation of u0 stay ordinary torch code.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np
import torch

from . import capi
from .workloads import SplitMix64


class Adjoint:
    """Checkpointed forward / backward of nsteps steps on one grid."""

    def __init__(self, shape, nsteps, dtype="f64", flux="hllc", gamma=1.4, boundary_mask=0,
                 interval=0, flatten=True, recon="muscl", p_inf=0.0):
        self.lib = capi.load()
        self.shape = tuple(int(v) for v in shape)
        self.nsteps = int(nsteps)
        self.gamma = float(gamma)
        self.policy = capi.policy_bits(dtype, flux, recon=recon, flatten=flatten)
        self.grid = capi.Grid.make(self.shape)
        self.dtype = torch.float64 if dtype == "f64" else torch.float32
        h = C.c_void_p()
        capi.check(self.lib.fl_adj_create(C.byref(h), C.byref(self.grid), self.gamma,
                                          self.policy, int(boundary_mask), self.nsteps,
                                          int(interval)), self.lib)
        self.handle = h
        self.p_inf = float(p_inf)
        if self.p_inf != 0.0:
            mat = capi.Material(self.gamma, self.p_inf)
            capi.check(self.lib.fl_adj_set_material(h, C.byref(mat)), self.lib)

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            try:
                self.lib.fl_adj_destroy(h)
            except Exception:
                pass
            self.handle = None

    @staticmethod
    def _s():
        return C.c_void_p(torch.cuda.current_stream().cuda_stream)

    def forward(self, u0, cfl=0.7, res=None, frozen_dtdh=None):
        """u_N from u0 ((dims + 2, cells) cuda tensor).  With frozen_dtdh (a
        sequence of nsteps dt/dh values) the steps replay those time steps."""
        res = 1.0 / self.shape[0] if res is None else res
        u0 = u0.contiguous()
        out = torch.empty_like(u0)
        fz = None
        if frozen_dtdh is not None:
            arr = np.ascontiguousarray(frozen_dtdh, dtype=np.float64)
            assert arr.size == self.nsteps
            fz = arr.ctypes.data_as(C.POINTER(C.c_double))
            self._keep = arr
        capi.check(self.lib.fl_adj_forward(self.handle, C.c_void_p(u0.data_ptr()),
                                           C.c_void_p(out.data_ptr()), float(cfl), float(res),
                                           fz, self._s()), self.lib)
        return out

    def dtdh(self):
        out = np.empty(self.nsteps, dtype=np.float64)
        capi.check(self.lib.fl_adj_dtdh(self.handle, out.ctypes.data_as(C.POINTER(C.c_double))),
                   self.lib)
        return out

    def backward(self, lam_final):
        lam_final = lam_final.contiguous()
        lam0 = torch.empty_like(lam_final)
        capi.check(self.lib.fl_adj_backward(self.handle, C.c_void_p(lam_final.data_ptr()),
                                            C.c_void_p(lam0.data_ptr()), self._s()), self.lib)
        return lam0


class EulerRollout(torch.autograd.Function):
    """u_N = rollout(u0); backward by the hand-written discrete adjoint."""

    @staticmethod
    def forward(ctx, u0, adj: Adjoint, cfl, res, frozen_dtdh):
        ctx.adj = adj
        return adj.forward(u0.detach(), cfl, res, frozen_dtdh)

    @staticmethod
    def backward(ctx, grad_out):
        return ctx.adj.backward(grad_out), None, None, None, None


def rollout(u0, adj: Adjoint, cfl=0.7, res=None, frozen_dtdh=None):
    return EulerRollout.apply(u0, adj, cfl, res, frozen_dtdh)


# ---- the gradient workload: smooth density, objective on the pressure ------

def gaussian_density(n: int, seed: int, count: int = 32, device="cuda",
                     dtype=torch.float64):
    """rho0 = 1 + sum of `count` Gaussians (amplitude in [0.1, 1], width in
    [0.02, 0.1], centres uniform in [0, 1]^2) at cell centres of an n x n grid;
    returns (n * n,) with x fastest."""
    rng = SplitMix64(seed)
    x = (torch.arange(n, device=device, dtype=dtype) + 0.5) / n
    X = x.repeat(n)
    Y = x.repeat_interleave(n)
    rho = torch.ones(n * n, device=device, dtype=dtype)
    for _ in range(count):
        amp = rng.uniform(0.1, 1.0)
        w = rng.uniform(0.02, 0.1)
        cx, cy = rng.uniform(0.0, 1.0), rng.uniform(0.0, 1.0)
        rho = rho + amp * torch.exp(-((X - cx) ** 2 + (Y - cy) ** 2) / (2 * w * w))
    return rho


def state_from_density(rho, gamma=1.4, temperature=1.0):
    """Conservative state at rest with p = rho * temperature:
    [rho, rho * temperature / (gamma - 1), 0, 0].  (A uniform pressure at rest
    would be an exact steady state -- every cell a stationary contact, which
    MUSCL-Hancock with HLLC keeps exactly -- so nothing would move and a
    pressure objective would not depend on the density.)"""
    E = rho * (temperature / (gamma - 1.0))
    z = torch.zeros_like(rho)
    return torch.stack([rho, E, z, z])


def pressure(u, gamma=1.4):
    rho = u[0]
    ke = 0.5 * (u[2] * u[2] + u[3] * u[3]) / rho
    return (gamma - 1.0) * (u[1] - ke)


def objective(u_final, p_target, gamma=1.4):
    """J = 0.5 ||p(T) - p_target||^2."""
    d = pressure(u_final, gamma) - p_target
    return 0.5 * torch.sum(d * d)


def objective_difference(u_plus, u_minus, p_target, gamma=1.4):
    """J(u_plus) - J(u_minus) without forming either J: the sum of
    0.5 (p+ - p-)(p+ + p- - 2 p_target) over cells.  A central difference
    of J itself loses about log10(J / dJ) digits to cancellation (J is
    O(1e5) on the 1024^2 workload while a directional derivative is O(1))."""
    pp = pressure(u_plus, gamma)
    pm = pressure(u_minus, gamma)
    return 0.5 * torch.sum((pp - pm) * (pp + pm - 2.0 * p_target))


def random_directions(n_cells: int, count: int, seed: int, device="cuda",
                      dtype=torch.float64):
    """Seeded unit directions for the finite-difference check."""
    g = torch.Generator(device="cpu").manual_seed(seed)
    v = torch.randn(count, n_cells, generator=g, dtype=torch.float64)
    v = v / v.norm(dim=1, keepdim=True)
    return v.to(device=device, dtype=dtype)
