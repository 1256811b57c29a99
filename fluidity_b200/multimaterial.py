"""Two-material ghost-fluid path on one GPU (fl_mm_* of the C ABI).

Mirrors the reference's MultimaterialSimulator
(simulator/multimaterial_simulator.hpp): two materials share a 2-D grid, each
with its own state buffers, equation of state (ideal gas, or the stiffened
fluid when its p_inf > 0) and FP64 level set; a step loads
the ghost cells (Riemann GFM + extrapolation), takes one CFL time step over
both materials, advances each material with the split solver and moves,
projects and reinitialises the level sets.  Device buffers are torch tensors
(plumbing only); all arithmetic is in libfluidity_b200.so.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import capi
from .solver import _stream_ptr

_DT = {"f64": torch.float64, "f32": torch.float32}


class MultiMaterial:
    def __init__(self, shape, gammas, res: float, dtype: str = "f32", flux: str = "hllc",
                 limiter: str = "vanleer", device="cuda", p_infs=(0.0, 0.0)):
        if len(shape) != 2:
            raise ValueError("the two-material path is 2-D")
        self.shape = tuple(int(v) for v in shape)
        self.cells = self.shape[0] * self.shape[1]
        self.dtype = dtype
        self.res = float(res)
        self.gammas = (float(gammas[0]), float(gammas[1]))
        self.p_infs = (float(p_infs[0]), float(p_infs[1]))
        self.materials = [capi.Material(g, p) for g, p in zip(self.gammas, self.p_infs)]
        self.policy = capi.policy_bits(dtype, flux, limiter)
        self.grid = capi.Grid.make(self.shape)
        self.lib = capi.load()
        g = (C.c_double * 2)(*self.gammas)
        h = C.c_void_p()
        capi.check(self.lib.fl_mm_create(C.byref(h), C.byref(self.grid), g, self.policy,
                                         self.res), self.lib)
        self.handle = h
        if any(self.p_infs):
            mats = (capi.Material * 2)(*self.materials)
            capi.check(self.lib.fl_mm_set_materials(h, mats), self.lib)
        dev = torch.device(device)
        self.u = [[torch.zeros((4, self.cells), dtype=_DT[dtype], device=dev) for _ in range(2)]
                  for _ in range(2)]
        self.phi = [[torch.zeros(self.cells, dtype=torch.float64, device=dev) for _ in range(2)]
                    for _ in range(2)]
        self._phi_by_ptr = {t.data_ptr(): t for pair in self.phi for t in pair}

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            try:
                self.lib.fl_mm_destroy(h)
            except Exception:
                pass
            self.handle = None

    # -- set-up --------------------------------------------------------------
    def set_states(self, material: int, phi, prim, stream=None):
        """state::set_states: cells of `material`'s state where phi <= 0 take
        the primitive state prim = (rho, p, v_x, v_y)."""
        pr = (C.c_double * 4)(*[float(v) for v in prim])
        phi_t = phi if isinstance(phi, torch.Tensor) else torch.tensor(
            np.ascontiguousarray(phi, dtype=np.float64), device=self.u[0][0].device)
        rc = self.lib.fl_mm_set_states_mat(C.byref(self.grid), self.policy,
                                           C.c_void_p(self.u[material][0].data_ptr()),
                                           C.c_void_p(phi_t.data_ptr()), pr,
                                           C.byref(self.materials[material]),
                                           _stream_ptr(stream))
        capi.check(rc, self.lib)

    def set_levelsets(self, phi0, phi1):
        for m, p in enumerate((phi0, phi1)):
            self.phi[m][0].copy_(torch.as_tensor(np.ascontiguousarray(p, dtype=np.float64)))

    @classmethod
    def shock_bubble(cls, spec, dtype: str = "f32", **kw):
        """Initial data of workloads.shock_bubble: each material's buffer is
        filled everywhere with its own gas (material 0 shocked behind the
        shock), then the level sets are set."""
        mm = cls((spec["nx"], spec["ny"]), spec["gammas"], spec["h"], dtype=dtype, **kw)
        everywhere = torch.full((mm.cells,), -1.0, dtype=torch.float64,
                                device=mm.u[0][0].device)
        mm.set_states(0, everywhere, spec["ambient"])
        mm.set_states(0, spec["shock_phi"], spec["shocked"])
        mm.set_states(1, everywhere, spec["bubble"])
        mm.set_levelsets(spec["phi0"], spec["phi1"])
        return mm

    # -- single operations ---------------------------------------------------
    def ghost(self, max_iters: int = 64, stream=None):
        rc = self.lib.fl_mm_ghost(self.handle, C.c_void_p(self.u[0][0].data_ptr()),
                                  C.c_void_p(self.u[1][0].data_ptr()),
                                  C.c_void_p(self.u[0][1].data_ptr()),
                                  C.c_void_p(self.u[1][1].data_ptr()),
                                  C.c_void_p(self.phi[0][0].data_ptr()),
                                  C.c_void_p(self.phi[1][0].data_ptr()), int(max_iters),
                                  _stream_ptr(stream))
        capi.check(rc, self.lib)

    def combine(self, out=None, stream=None):
        """material::combine_into_first into a copy of material 0's state."""
        out = self.u[0][0].clone() if out is None else out
        phi1 = self.current_phi()[1]
        rc = self.lib.fl_mm_combine(C.byref(self.grid), self.policy, C.c_void_p(out.data_ptr()),
                                    C.c_void_p(self.u[1][0].data_ptr()),
                                    C.c_void_p(phi1.data_ptr()), _stream_ptr(stream))
        capi.check(rc, self.lib)
        return out

    def stats(self):
        out = (C.c_int32 * 8)()
        capi.check(self.lib.fl_mm_stats(self.handle, out, 8), self.lib)
        keys = ["gfm0", "gfm1", "band0", "band1", "extrap_iters0", "extrap_iters1",
                "reinit_passes0", "reinit_passes1"]
        return dict(zip(keys, list(out)))

    # -- step loop -----------------------------------------------------------
    def begin(self, cfl: float, sim_time: float, max_iters: int, reinit_every: int = 5):
        p = lambda t: C.c_void_p(t.data_ptr())
        rc = self.lib.fl_mm_begin(self.handle, p(self.u[0][0]), p(self.u[0][1]), p(self.u[1][0]),
                                  p(self.u[1][1]), p(self.phi[0][0]), p(self.phi[0][1]),
                                  p(self.phi[1][0]), p(self.phi[1][1]), float(cfl),
                                  float(sim_time), int(max_iters), int(reinit_every))
        capi.check(rc, self.lib)

    def steps(self, n: int, stream=None):
        capi.check(self.lib.fl_mm_steps(self.handle, int(n), _stream_ptr(stream)), self.lib)

    def status(self, stream=None):
        it = C.c_int64()
        rt = C.c_double()
        done = C.c_int()
        p0 = C.c_void_p()
        p1 = C.c_void_p()
        rc = self.lib.fl_mm_status(self.handle, _stream_ptr(stream), C.byref(it), C.byref(rt),
                                   C.byref(done), C.byref(p0), C.byref(p1))
        capi.check(rc, self.lib)
        return int(it.value), float(rt.value), bool(done.value)

    def current_phi(self):
        it = C.c_int64()
        rt = C.c_double()
        done = C.c_int()
        p0 = C.c_void_p()
        p1 = C.c_void_p()
        rc = self.lib.fl_mm_status(self.handle, None, C.byref(it), C.byref(rt), C.byref(done),
                                   C.byref(p0), C.byref(p1))
        capi.check(rc, self.lib)
        if not p0.value:   # before fl_mm_begin: buffer 0
            return self.phi[0][0], self.phi[1][0]
        return self._phi_by_ptr[p0.value], self._phi_by_ptr[p1.value]

    def states(self):
        return self.u[0][0], self.u[1][0]
