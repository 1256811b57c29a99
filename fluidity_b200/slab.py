"""One 2-D grid decomposed into slabs of rows, one rank (GPU) per slab.

The split step is local except along y: a sweep reads 4 rows beyond its own
along the sweep (MUSCL-Hancock with flattening) and 3 across it (the
flattening coefficient takes the minimum over both dimensions).  Each rank
therefore holds its rows plus GHOST = 4 ghost rows on every side that faces
another rank, and before each sweep it refreshes the rows that sweep reads
from its neighbours: ROWS_X = 3 before the x sweep, ROWS_Y = 4 before the y
sweep (two point-to-point exchanges per step, over NCCL on GPUs).  A ghost row's
own update is discarded: the next exchange overwrites it.  At the domain's
top and bottom a slab has no ghost rows and the kernels' mirror ghosts apply,
exactly as on the undivided grid.  The CFL maximum is reduced once per step
across ranks (a 64-bit MAX on the double's bits) before the control block
takes the next time step, so every rank steps with the same dt and the result
equals the undivided run's.

`SlabRunner` holds this schedule and is independent of where the sweeps run;
`CudaSlabOps` runs them with libfluidity_b200.so (fl_sim_sweep,
fl_sim_finalize, the wavespeed row window and the external reduction).
`NativeSlabs` enqueues the same schedule below the host (fl_slab_*): whole
steps in one call, over NCCL with one rank per GPU or over device copies for
slabs held by one process.
"""
from __future__ import annotations

import ctypes as C

import torch
import torch.distributed as dist

from . import capi

GHOST = 4
ROWS_X = 3   # ghost rows the x sweep reads
ROWS_Y = 4   # ghost rows the y sweep reads


def slab_rows(ny: int, world: int, rank: int) -> tuple[int, int]:
    """Own rows [lo, hi) of `rank`: an even split, the first ny % world
    ranks taking one row more."""
    base, extra = divmod(ny, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


class SlabLayout:
    """Local grid of one rank: own rows plus ghost rows facing neighbours."""

    def __init__(self, shape, world: int, rank: int, ghost: int = GHOST):
        self.nx, self.ny = int(shape[0]), int(shape[1])
        self.world, self.rank, self.ghost = world, rank, ghost
        self.lo, self.hi = slab_rows(self.ny, world, rank)
        if self.hi - self.lo < ghost:
            raise ValueError(f"slab of {self.hi - self.lo} rows is thinner than {ghost} ghost rows")
        self.g_bot = ghost if rank > 0 else 0
        self.g_top = ghost if rank < world - 1 else 0
        self.rows = self.hi - self.lo + self.g_bot + self.g_top
        self.row0 = self.lo - self.g_bot                 # global row of local row 0
        self.own = (self.g_bot, self.g_bot + self.hi - self.lo)   # local own rows

    @property
    def local_shape(self):
        return (self.nx, self.rows)

    @property
    def cells(self):
        return self.nx * self.rows

    def own_slice(self):
        """Flat cell range of the own rows in a local plane."""
        return slice(self.own[0] * self.nx, self.own[1] * self.nx)

    def global_slice(self):
        """Flat cell range of the local rows (ghosts included) in a global plane."""
        return slice(self.row0 * self.nx, (self.row0 + self.rows) * self.nx)


class SlabExchange:
    """Ghost-row exchange between neighbouring slabs: own boundary rows go
    out, the neighbour's boundary rows land in the ghost rows (every state
    plane, one send and one receive per neighbour and plane)."""

    def __init__(self, layout: SlabLayout, group=None):
        self.L = layout
        self.group = group

    def __call__(self, state: torch.Tensor, rows: int = GHOST):
        L, nx, g = self.L, self.L.nx, rows
        ops = []
        for c in range(state.shape[0]):
            plane = state[c]
            if L.rank > 0:
                ops.append(dist.P2POp(dist.isend, plane[L.own[0] * nx:(L.own[0] + g) * nx],
                                      L.rank - 1, self.group))
                ops.append(dist.P2POp(dist.irecv, plane[(L.own[0] - g) * nx:L.own[0] * nx],
                                      L.rank - 1, self.group))
            if L.rank < L.world - 1:
                ops.append(dist.P2POp(dist.isend, plane[(L.own[1] - g) * nx:L.own[1] * nx],
                                      L.rank + 1, self.group))
                ops.append(dist.P2POp(dist.irecv, plane[L.own[1] * nx:(L.own[1] + g) * nx],
                                      L.rank + 1, self.group))
        if ops:
            for req in dist.batch_isend_irecv(ops):
                req.wait()


class SlabRunner:
    """The decomposed time loop: exchange, sweep x, exchange, sweep y (the
    fused max wavespeed over own rows), MAX-reduce the wavespeed word,
    finalise the step.  `ops` runs the sweeps and owns the control block
    (CudaSlabOps on GPUs)."""

    def __init__(self, layout: SlabLayout, ops, group=None):
        self.L = layout
        self.ops = ops
        self.group = group
        self.exchange = SlabExchange(layout, group)

    def _reduce_ws(self):
        if self.L.world > 1:
            dist.all_reduce(self.ops.ws_word, op=dist.ReduceOp.MAX, group=self.group)

    def begin(self, a, b, cfl, res, sim_time, max_iters):
        self.ops.begin(a, b, cfl, res, sim_time, max_iters)
        self._reduce_ws()
        self.ops.finalize(advance=False)

    def step(self):
        a, b = self.ops.buffers
        self.exchange(a, ROWS_X)
        self.ops.sweep(0)     # a -> b
        self.exchange(b, ROWS_Y)
        self.ops.sweep(1)     # b -> a, wavespeed word over own rows
        self._reduce_ws()
        self.ops.finalize(advance=True)

    def steps(self, n: int):
        for _ in range(n):
            self.step()


class CudaSlabOps:
    """Sweeps and control of one slab on the current GPU (fl_sim in its
    external-reduction mode)."""

    def __init__(self, layout: SlabLayout, dtype="f64", flux="hllc", limiter="vanleer",
                 gamma=1.4, boundary_mask=0):
        from .solver import Simulation, SplitSolver, _stream_ptr
        self._stream = _stream_ptr
        self.solver = SplitSolver(layout.local_shape, dtype=dtype, flux=flux, limiter=limiter,
                                  gamma=gamma, boundary_mask=boundary_mask)
        self.sim = Simulation(self.solver)
        self.lib = self.solver.lib
        self.ws_word = torch.zeros(1, dtype=torch.int64, device="cuda")
        h = self.sim.handle
        capi.check(self.lib.fl_sim_set_rows(h, layout.own[0], layout.own[1]), self.lib)
        capi.check(self.lib.fl_sim_set_external_reduce(h, 1), self.lib)
        capi.check(self.lib.fl_sim_set_ws_word(h, C.c_void_p(self.ws_word.data_ptr())), self.lib)
        self.buffers = None

    def new_state(self):
        return self.solver.new_state()

    def begin(self, a, b, cfl, res, sim_time, max_iters):
        self.buffers = (a, b)
        self.sim.begin(a, b, cfl, res, sim_time, max_iters)

    def sweep(self, dim):
        capi.check(self.lib.fl_sim_sweep(self.sim.handle, int(dim), self._stream()), self.lib)

    def finalize(self, advance):
        capi.check(self.lib.fl_sim_finalize(self.sim.handle, int(bool(advance)), self._stream()),
                   self.lib)

    def status(self, allow_nan=False):
        return self.sim.status(allow_nan=allow_nan)


class NativeSlabs:
    """Slabs of one grid stepped below the host (fl_slab_* in
    include/fluidity_b200.h): one call enqueues whole steps -- exchange
    ROWS_X rows, x sweep, exchange ROWS_Y rows, y sweep, wavespeed maximum
    over the slabs, finalize -- on the current stream.

    ``NativeSlabs.local(layouts, ...)``: every slab in this process, in
    order, exchanged by device copies.  ``NativeSlabs.nccl(layout, ...)``:
    this rank's slab of a torch.distributed job, exchanged over an NCCL
    communicator of its own (the id is broadcast over the default group)."""

    def __init__(self, layouts, handles, lib, dtype):
        self.layouts = layouts
        self.handles = handles
        self.lib = lib
        self.dtype = dtype
        self._arr = (C.c_void_p * len(handles))(*handles)
        self.buffers = None

    @classmethod
    def local(cls, layouts, dtype="f64", flux="hllc", limiter="vanleer", gamma=1.4):
        lib = capi.load()
        pol = capi.policy_bits(dtype, flux, limiter)
        hs = []
        try:
            for L in layouts:
                h = C.c_void_p()
                g = capi.Grid.make(L.local_shape)
                capi.check(lib.fl_slab_create_local(C.byref(h), C.byref(g), gamma, pol, 0,
                                                    L.own[0], L.own[1]), lib)
                hs.append(h.value)
        except Exception:
            for h in hs:
                lib.fl_slab_destroy(h)
            raise
        return cls(list(layouts), hs, lib, dtype)

    @classmethod
    def nccl(cls, layout, dtype="f64", flux="hllc", limiter="vanleer", gamma=1.4, group=None):
        lib = capi.load()
        pol = capi.policy_bits(dtype, flux, limiter)
        idbuf = (C.c_char * 128)()
        if layout.world == 1:
            capi.check(lib.fl_slab_nccl_id(idbuf), lib)   # a communicator of one rank
        else:
            if not lib.fl_slab_nccl_available():
                raise RuntimeError("libnccl.so.2 could not be loaded")
            obj = [None]
            if layout.rank == 0:
                capi.check(lib.fl_slab_nccl_id(idbuf), lib)
                obj = [bytes(idbuf)]
            dist.broadcast_object_list(obj, src=0, group=group)
            C.memmove(idbuf, obj[0], 128)
        h = C.c_void_p()
        g = capi.Grid.make(layout.local_shape)
        capi.check(lib.fl_slab_create_nccl(C.byref(h), C.byref(g), gamma, pol, 0, layout.own[0],
                                           layout.own[1], idbuf, layout.world, layout.rank), lib)
        return cls([layout], [h.value], lib, dtype)

    def new_state(self, i=0):
        L = self.layouts[i]
        tdt = torch.float64 if self.dtype == "f64" else torch.float32
        return torch.zeros((4, L.cells), dtype=tdt, device="cuda")

    def _stream(self):
        return C.c_void_p(torch.cuda.current_stream().cuda_stream)

    def begin(self, a, b, cfl, res, sim_time, max_iters):
        """a[i], b[i]: slab i's buffers, a[i] holding its initial state
        (ghost rows included)."""
        self.buffers = (list(a), list(b))
        pa = (C.c_void_p * len(a))(*[t.data_ptr() for t in a])
        pb = (C.c_void_p * len(b))(*[t.data_ptr() for t in b])
        capi.check(self.lib.fl_slab_begin(self._arr, len(self.handles), pa, pb, cfl, res,
                                          sim_time, max_iters, self._stream()), self.lib)

    def steps(self, n: int):
        capi.check(self.lib.fl_slab_steps(self._arr, len(self.handles), int(n), self._stream()),
                   self.lib)

    def status(self, i=0):
        sim = C.c_void_p()
        capi.check(self.lib.fl_slab_sim(self.handles[i], C.byref(sim)), self.lib)
        it, rt, done, res = C.c_int64(), C.c_double(), C.c_int(), C.c_void_p()
        capi.check(self.lib.fl_sim_status(sim, self._stream(), C.byref(it), C.byref(rt),
                                          C.byref(done), C.byref(res)), self.lib)
        return it.value, rt.value, bool(done.value)

    def close(self):
        for h in self.handles:
            self.lib.fl_slab_destroy(h)
        self.handles = []

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
