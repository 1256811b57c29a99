"""Level-set operations of the multimaterial (ghost-fluid) path on one GPU.

Thin host mirror of the reference's level-set calls, each one C-ABI call
into libfluidity_b200.so:

* ``velocity``   -- set_velocities (levelset/cuda/velocity_initialization.cuh:108-143)
* ``advect``     -- one RK3 step of the level-set equation with WENO-HJ5 and
  the Godunov upwind Hamiltonian (scheme/cuda/evolve.cuh:51-157,
  scheme/updaters/runge_kutta_3.hpp:110-148)
* ``project``    -- two-material projection (levelset/cuda/levelset_projection.cuh:54-67)
* ``reinit``     -- fast-iterative-method reinitialisation
  (scheme/cuda/fast_iterative_method.cuh:48-112)

FP64 level sets, 2-D grids, x fastest.  The workspace is allocated once per
grid; no call allocates device memory.
"""
from __future__ import annotations

import ctypes as C

import torch

from . import capi
from .solver import _stream_ptr


class LevelSetOps:
    def __init__(self, shape, device="cuda"):
        if len(shape) != 2:
            raise ValueError("level-set operations are 2-D")
        self.shape = tuple(int(v) for v in shape)
        self.cells = self.shape[0] * self.shape[1]
        self.grid = capi.Grid.make(self.shape)
        self.lib = capi.load()
        nbytes = self.lib.fl_ls_workspace_bytes(C.byref(self.grid))
        if nbytes < 0:
            capi.check(capi.FL_EINVAL, self.lib)
        self.workspace = torch.empty(int(nbytes), dtype=torch.uint8, device=device)
        self.passes = 0

    def new(self):
        return torch.empty(self.cells, dtype=torch.float64, device=self.workspace.device)

    def velocity(self, phis, states, h: float, dtype: str = "f64", out=None, stream=None):
        """Interface-normal velocity of the first material (of 1 or 2) that
        contains each cell; states are SoA (4, pitch) tensors."""
        out = self.new() if out is None else out
        n = len(phis)
        pp = (C.c_void_p * n)(*[p.data_ptr() for p in phis])
        sp = (C.c_void_p * n)(*[s.data_ptr() for s in states])
        pol = capi.policy_bits(dtype)
        rc = self.lib.fl_ls_velocity(C.byref(self.grid), n, pp, sp, int(states[0].shape[1]), pol,
                                     float(h), C.c_void_p(out.data_ptr()), _stream_ptr(stream))
        capi.check(rc, self.lib)
        return out

    def advect(self, phi, vel, dt: float, h: float, out=None, stream=None):
        out = self.new() if out is None else out
        rc = self.lib.fl_ls_advect(C.byref(self.grid), C.c_void_p(phi.data_ptr()),
                                   C.c_void_p(vel.data_ptr()), float(dt), float(h),
                                   C.c_void_p(out.data_ptr()),
                                   C.c_void_p(self.workspace.data_ptr()), _stream_ptr(stream))
        capi.check(rc, self.lib)
        return out

    def project(self, a, b, stream=None):
        rc = self.lib.fl_ls_project(a.numel(), C.c_void_p(a.data_ptr()), C.c_void_p(b.data_ptr()),
                                    _stream_ptr(stream))
        capi.check(rc, self.lib)

    def reinit(self, phi, h: float, out=None, max_passes: int = 100000, stream=None):
        out = self.new() if out is None else out
        passes = C.c_int()
        rc = self.lib.fl_ls_reinit(C.byref(self.grid), C.c_void_p(phi.data_ptr()), float(h),
                                   C.c_void_p(out.data_ptr()),
                                   C.c_void_p(self.workspace.data_ptr()), int(max_passes),
                                   C.byref(passes), _stream_ptr(stream))
        self.passes = int(passes.value)
        capi.check(rc, self.lib)
        return out
