"""The slab decomposition's schedule on CPU ranks (gloo): ghost-row exchange
before every sweep, the CFL maximum reduced over ranks, the step finalised
from it.  The oracle performs the sweeps here (it applies the same mirror
rule at a slab's outer rows as the CUDA kernels do), so the decomposed run
must reproduce the undivided oracle run bit for bit.  On GPUs the same
SlabRunner drives the CUDA sweeps and NCCL (fluidity_b200.slab.CudaSlabOps).
"""
import os
import socket
import struct

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

GAMMA = 1.4


def _bits(x: float) -> int:
    return struct.unpack("<q", struct.pack("<d", float(x)))[0]


def _from_bits(b: int) -> float:
    return struct.unpack("<d", struct.pack("<q", int(b)))[0]


class OracleSlabOps:
    """CPU stand-in for CudaSlabOps: oracle sweeps on the local grid and the
    FP64 control arithmetic of the device time loop (dt = cfl*dh/ws,
    dtdh = dt/dh, run_time += dt, stop test)."""

    def __init__(self, layout, flux="hllc"):
        from oracle import oracle
        self.O = oracle
        self.L = layout
        self.flux = flux
        self.ws_word = torch.zeros(1, dtype=torch.int64)
        self.buffers = None

    def _own_ws(self, u):
        L = self.L
        own = u[:, L.own_slice()].numpy()
        return self.O.max_wavespeed((L.nx, L.own[1] - L.own[0]), np.ascontiguousarray(own),
                                    GAMMA)

    def begin(self, a, b, cfl, res, sim_time, max_iters):
        self.buffers = (a, b)
        self.cfl, self.res, self.sim_time, self.max_iters = cfl, res, sim_time, max_iters
        self.run_time, self.iters, self.done, self.dt, self.dtdh = 0.0, 0, False, 0.0, 0.0
        self.ws_word[0] = _bits(self._own_ws(a))

    def sweep(self, dim):
        a, b = self.buffers
        src, dst = (a, b) if dim == 0 else (b, a)
        if self.done:
            return
        out = self.O.sweep(self.L.local_shape, dim, src.numpy(), GAMMA, self.dtdh, flux=self.flux)
        dst.copy_(torch.from_numpy(out))
        if dim == 1:
            self.ws_word[0] = _bits(self._own_ws(dst))

    def finalize(self, advance):
        if self.done:
            return
        ws = _from_bits(int(self.ws_word[0]))
        self.ws_word[0] = 0
        if advance:
            self.run_time = self.run_time + self.dt
            self.iters += 1
        self.dt = self.cfl * self.res / ws
        self.dtdh = self.dt / self.res
        self.done = not (self.run_time < self.sim_time and self.iters < self.max_iters)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _poisoning_runner(SlabRunner, ROWS_X, ROWS_Y):
    """SlabRunner whose x sweep sees a strong pressure jump (rho 1, E 1e4,
    at rest) in every ghost row the x exchange does not refresh: the
    flattening coefficient reacts to it, so the result can only stay exact if
    the x sweep never reads those rows.  (NaN would not do: the coefficient's
    comparisons are false for NaN and leave it unflattened.)"""

    class Poisoned(SlabRunner):
        def step(self):
            a, b = self.ops.buffers
            L, nx = self.L, self.L.nx
            self.exchange(a, ROWS_X)
            for lo, hi in ((0, L.own[0] - ROWS_X), (L.own[1] + ROWS_X, L.rows)):
                if hi > lo:
                    a[:, lo * nx:hi * nx] = 0.0
                    a[0, lo * nx:hi * nx] = 1.0
                    a[1, lo * nx:hi * nx] = 1e4
            self.ops.sweep(0)
            self.exchange(b, ROWS_Y)
            self.ops.sweep(1)
            self._reduce_ws()
            self.ops.finalize(advance=True)

    return Poisoned


def _rank_main(rank, world, port, shape, u0, nsteps, out_path, poison=False):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from fluidity_b200.slab import ROWS_X, ROWS_Y, SlabLayout, SlabRunner
        if poison:
            SlabRunner = _poisoning_runner(SlabRunner, ROWS_X, ROWS_Y)
        L = SlabLayout(shape, world, rank)
        ops = OracleSlabOps(L)
        a = torch.from_numpy(np.ascontiguousarray(u0[:, L.global_slice()]))
        b = torch.zeros_like(a)
        run = SlabRunner(L, ops)
        run.begin(a, b, 0.8, 1.0 / shape[0], 1e30, nsteps)
        run.steps(nsteps)
        own = a[:, L.own_slice()].clone()
        parts = [None] * world
        dist.all_gather_object(parts, (L.lo, L.hi, own.numpy(), ops.iters, ops.run_time))
        if rank == 0:
            np.save(out_path, np.array(parts, dtype=object), allow_pickle=True)
    finally:
        dist.destroy_process_group()


def _run(world, shape, nsteps, tmp_path, poison=False):
    from _util import random_prim
    from oracle import oracle
    prim = random_prim(shape, 5, smooth=True, mild=True)
    u0 = oracle.prim_to_cons(prim, GAMMA)
    out = str(tmp_path / f"slab_{world}.npy")
    mp.start_processes(_rank_main, args=(world, _free_port(), shape, u0, nsteps, out, poison),
                       nprocs=world, join=True, start_method="spawn")
    parts = np.load(out, allow_pickle=True)
    got = np.zeros_like(u0)
    nx = shape[0]
    for lo, hi, own, iters, rt in parts:
        got[:, lo * nx:hi * nx] = own
        assert iters == nsteps
    want, steps, run_time, _ = oracle.simulate(shape, u0, GAMMA, 0.8, 1.0 / shape[0], 1e30,
                                               nsteps)
    assert steps == nsteps
    assert all(rt == run_time for *_, rt in parts)
    return got, want


@pytest.mark.parametrize("world", [2, 3])
def test_slab_decomposition_matches_undivided_run(world, tmp_path):
    got, want = _run(world, (24, 37), 6, tmp_path)
    assert np.array_equal(got, want)


def test_x_sweep_reads_three_ghost_rows(tmp_path):
    """3 ghost rows before the x sweep are enough: with the fourth poisoned
    before every x sweep the decomposed run still equals the undivided one.
    (3 across and 4 along are the stencil's bounds; on random states a
    changed row was seen to move x-sweep results at most 2 rows away and
    y-sweep results at most 3.)"""
    got, want = _run(3, (24, 37), 5, tmp_path, poison=True)
    assert np.array_equal(got, want)


def test_slab_rows_cover_the_grid():
    from fluidity_b200.slab import SlabLayout, slab_rows
    for ny, world in ((37, 3), (4096, 8), (100, 7)):
        spans = [slab_rows(ny, world, r) for r in range(world)]
        assert spans[0][0] == 0 and spans[-1][1] == ny
        assert all(spans[i][1] == spans[i + 1][0] for i in range(world - 1))
        assert max(h - l for l, h in spans) - min(h - l for l, h in spans) <= 1
    L = SlabLayout((16, 37), 3, 1)
    assert (L.g_bot, L.g_top, L.rows) == (4, 4, L.hi - L.lo + 8)
    L0 = SlabLayout((16, 37), 3, 0)
    assert L0.g_bot == 0 and L0.row0 == 0
    with pytest.raises(ValueError):
        SlabLayout((16, 10), 4, 0)
