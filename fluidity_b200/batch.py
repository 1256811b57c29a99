"""Batched solver: thousands of independent 1-D / 2-D Riemann problems in
one persistent launch per size class (1-D, resident in shared memory) and one
batched launch per sweep (2-D), with the time loop captured in a CUDA graph
and tile shapes picked by the autotuner (fl_batch_* in include/fluidity_b200.h).

The problem states live in two torch arenas; problem i's planes start at
``offsets[i]`` with pitch ``pitches[i]`` (cells rounded up to 32 elements so
that every plane starts 128-byte aligned).
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np
import torch

from . import capi
from .workloads import SplitMix64, riemann_states


def batched_workload(seed: int = 3, n1d: int = 3584, n2d: int = 512, lo1=64, hi1=8192,
                     lo2=64, hi2=512):
    """Problem sizes and initial primitive states of the batched workload:
    n1d 1-D problems with cell counts log-uniform in [lo1, hi1] and n2d 2-D
    problems with sides log-uniform in [lo2, hi2]; each problem's states come
    from riemann_states (rho in [0.1, 10], |v| <= 2, p in [0.01, 1000])."""
    rng = SplitMix64(seed)
    problems = []
    for i in range(n1d + n2d):
        if i < n1d:
            n = int(round(math.exp(rng.uniform(math.log(lo1), math.log(hi1)))))
            problems.append(((n,), riemann_states(rng.next_u64(), 1)))
        else:
            s = int(round(math.exp(rng.uniform(math.log(lo2), math.log(hi2)))))
            problems.append(((s, s), riemann_states(rng.next_u64(), 2)))
    return problems


def problem_cost(shape) -> int:
    """Work of one time step of a problem: cells x sweeps (one sweep per
    dimension).  For a run of a fixed step count this orders problems by
    their device time."""
    return int(np.prod(shape)) * len(shape)


def partition_problems(problems, world: int) -> list[list[int]]:
    """Cost-balanced split of a problem list over `world` ranks (one GPU
    each), with no communication: every rank computes the same split.

    Greedy longest-first: problems in decreasing cost (ties by index) go
    one by one to the rank with the least cost so far (ties to the lowest
    rank).  The largest load exceeds the smallest by at most one problem's
    cost.  Returns, per rank, the problem indices in increasing order."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(problems)), key=lambda i: (-problem_cost(problems[i][0]), i))
    load = [0] * world
    parts: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        parts[r].append(i)
        load[r] += problem_cost(problems[i][0])
    return [sorted(p) for p in parts]


class Batch:
    """A set of problems, their arenas and the fl_batch handle."""

    def __init__(self, problems, dtype: str = "f32", flux: str = "hllc", gamma: float = 1.4,
                 boundary_mask: int = 0, device="cuda", p_inf: float = 0.0):
        self.lib = capi.load()
        self.problems = problems
        self.dtype = dtype
        self.gamma = gamma
        self.policy = capi.policy_bits(dtype, flux)
        tdt = torch.float32 if dtype == "f32" else torch.float64
        descs = (capi.BatchDesc * len(problems))()
        off = 0
        self.offsets, self.pitches = [], []
        for i, (shape, _) in enumerate(problems):
            cells = int(np.prod(shape))
            pitch = (cells + 31) // 32 * 32
            d = descs[i]
            d.dims = len(shape)
            d.n[0] = shape[0]
            d.n[1] = shape[1] if len(shape) > 1 else 1
            d.offset = off
            d.pitch = pitch
            d.res = 1.0 / shape[0]
            self.offsets.append(off)
            self.pitches.append(pitch)
            off += (len(shape) + 2) * pitch
        self.total = off
        self.cells = sum(int(np.prod(s)) for s, _ in problems)
        self.a = torch.zeros(off, dtype=tdt, device=device)
        self.b = torch.zeros(off, dtype=tdt, device=device)
        h = C.c_void_p()
        capi.check(self.lib.fl_batch_create(C.byref(h), descs, len(problems), gamma,
                                            self.policy, boundary_mask), self.lib)
        self.handle = h
        self.p_inf = float(p_inf)
        if self.p_inf != 0.0:
            mat = capi.Material(float(gamma), self.p_inf)
            capi.check(self.lib.fl_batch_set_material(h, C.byref(mat)), self.lib)

    @classmethod
    def shard(cls, problems, world: int, rank: int, **kw):
        """This rank's share of a batch split over `world` GPUs by
        partition_problems: (Batch of the share, the share's indices into
        `problems`).  No collective is involved."""
        idx = partition_problems(problems, world)[rank]
        return cls([problems[i] for i in idx], **kw), idx

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            try:
                self.lib.fl_batch_destroy(h)
            except Exception:
                pass
            self.handle = None

    def fill(self):
        """Writes every problem's Riemann initial state into arena a."""
        for i, (shape, states) in enumerate(self.problems):
            g = capi.Grid.make(shape, self.pitches[i])
            elem = self.a.element_size()
            ptr = self.a.data_ptr() + self.offsets[i] * elem
            sp = np.ascontiguousarray(states, dtype=np.float64)
            if self.p_inf != 0.0:
                mat = capi.Material(float(self.gamma), self.p_inf)
                rc = self.lib.fl_fill_riemann_mat(C.byref(g), sp.ctypes.data_as(C.c_void_p),
                                                  C.byref(mat), self.policy, C.c_void_p(ptr),
                                                  None)
            else:
                rc = self.lib.fl_fill_riemann(C.byref(g), sp.ctypes.data_as(C.c_void_p),
                                              self.gamma, self.policy, C.c_void_p(ptr), None)
            capi.check(rc, self.lib)

    def state(self, i, arena=None):
        arena = self.a if arena is None else arena
        shape = self.problems[i][0]
        cells = int(np.prod(shape))
        o, p = self.offsets[i], self.pitches[i]
        return arena[o:o + (len(shape) + 2) * p].view(len(shape) + 2, p)[:, :cells]

    def _s(self, stream):
        s = stream if stream is not None else torch.cuda.current_stream()
        return C.c_void_p(s.cuda_stream)

    def begin(self, cfl=0.8, sim_time=1e30, max_iters=200, stream=None):
        capi.check(self.lib.fl_batch_begin(self.handle, C.c_void_p(self.a.data_ptr()),
                                           C.c_void_p(self.b.data_ptr()), cfl, sim_time,
                                           int(max_iters), self._s(stream)), self.lib)

    def steps(self, n, stream=None):
        capi.check(self.lib.fl_batch_steps(self.handle, int(n), self._s(stream)), self.lib)

    def capture(self, n):
        capi.check(self.lib.fl_batch_capture(self.handle, int(n)), self.lib)

    def launch(self, stream=None):
        capi.check(self.lib.fl_batch_launch(self.handle, self._s(stream)), self.lib)

    def status(self, stream=None, allow_nan=False):
        n = len(self.problems)
        it = (C.c_int64 * n)()
        rt = (C.c_double * n)()
        done = C.c_int32()
        rc = self.lib.fl_batch_status(self.handle, self._s(stream), it, rt, C.byref(done))
        if rc != capi.FL_OK and not (allow_nan and rc == capi.FL_ENAN):
            capi.check(rc, self.lib)
        return np.array(it[:]), np.array(rt[:]), int(done.value), rc

    def autotune(self, trial_steps=8, stream=None):
        capi.check(self.lib.fl_batch_autotune(self.handle, C.c_void_p(self.a.data_ptr()),
                                              C.c_void_p(self.b.data_ptr()), int(trial_steps),
                                              self._s(stream)), self.lib)
        return self.tuning()

    def tuning(self):
        out = (C.c_int32 * 8)()
        capi.check(self.lib.fl_batch_tuning(self.handle, out, 8), self.lib)
        v = list(out)
        return {"threads_1d": v[0:3], "class_bounds_1d": v[3:5], "strip_rows_2d": v[5:8]}
