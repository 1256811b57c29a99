"""The CUDA side of the slab decomposition on one GPU: two or three slabs of
one grid held by one process, stepped with fl_sim_sweep / fl_sim_finalize in
the decomposed schedule (the ghost-row exchange done by device copies
between the slabs' buffers, the CFL maximum by the largest of the slabs'
wavespeed words).  Launches are sequential and no kernel waits on another.
The result must equal the undivided run of the same grid bit for bit."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _exchange(layouts, bufs):
    """Ghost rows of each slab from its neighbours' own rows."""
    for r, L in enumerate(layouts):
        nx, g = L.nx, L.ghost
        if r > 0:
            P = layouts[r - 1]
            bufs[r][:, 0:g * nx] = bufs[r - 1][:, (P.own[1] - g) * nx:P.own[1] * nx]
        if r < len(layouts) - 1:
            N = layouts[r + 1]
            bufs[r][:, L.rows * nx - g * nx:L.rows * nx] = \
                bufs[r + 1][:, N.own[0] * nx:(N.own[0] + g) * nx]


def _reduce(ops):
    m = max(int(op.ws_word.item()) for op in ops)
    for op in ops:
        op.ws_word.fill_(m)


@pytest.mark.parametrize("dtype,world,shape", [("f64", 2, (96, 72)), ("f32", 3, (64, 45))])
def test_slabs_match_undivided_run(cuda, dtype, world, shape):
    from fluidity_b200.slab import CudaSlabOps, SlabLayout
    from fluidity_b200.solver import Simulation, SplitSolver
    from fluidity_b200.workloads import riemann_states
    T = 8
    full = SplitSolver(shape, dtype=dtype)
    u0 = full.fill_riemann(riemann_states(2, 2))
    sim = Simulation(full)
    want, it, rt = sim.run(u0.clone(), full.new_state(), 0.8, 1.0 / shape[0], 1e30, T)
    want = want.cpu().numpy()
    assert it == T

    layouts = [SlabLayout(shape, world, r) for r in range(world)]
    ops = [CudaSlabOps(L, dtype=dtype) for L in layouts]
    a = [u0[:, L.global_slice()].contiguous() for L in layouts]
    b = [op.new_state() for op in ops]
    for r in range(world):
        ops[r].begin(a[r], b[r], 0.8, 1.0 / shape[0], 1e30, T)
    _reduce(ops)
    for op in ops:
        op.finalize(advance=False)
    for _ in range(T):
        _exchange(layouts, a)
        for op in ops:
            op.sweep(0)
        _exchange(layouts, b)
        for op in ops:
            op.sweep(1)
        _reduce(ops)
        for op in ops:
            op.finalize(advance=True)
    got = np.zeros_like(want)
    nx = shape[0]
    for L, op, ar in zip(layouts, ops, a):
        its, rts, done, _ = op.status()
        assert its == T and done and rts == rt
        got[:, L.lo * nx:L.hi * nx] = ar[:, L.own_slice()].cpu().numpy()
    assert np.array_equal(got, want)


def _undivided(dtype, shape, T):
    from fluidity_b200.solver import Simulation, SplitSolver
    from fluidity_b200.workloads import riemann_states
    full = SplitSolver(shape, dtype=dtype)
    u0 = full.fill_riemann(riemann_states(2, 2))
    want, it, rt = Simulation(full).run(u0.clone(), full.new_state(), 0.8, 1.0 / shape[0], 1e30,
                                        T)
    assert it == T
    return u0, want.cpu().numpy(), rt


def _gather(layouts, bufs, like):
    got = np.zeros_like(like)
    for L, a in zip(layouts, bufs):
        got[:, L.lo * L.nx:L.hi * L.nx] = a[:, L.own_slice()].cpu().numpy()
    return got


@pytest.mark.parametrize("dtype,world,shape", [("f64", 2, (96, 72)), ("f32", 3, (64, 45)),
                                               ("f64", 4, (40, 64)), ("f64", 8, (32, 40))])
def test_native_slab_steps_match_undivided_run(cuda, dtype, world, shape):
    """fl_slab_steps with in-process slabs: the whole decomposed step (3-row
    exchange, x sweep, 4-row exchange, y sweep, wavespeed maximum, finalize)
    enqueued by one call, each sweep in parts (the rows that need no ghost
    row while the exchange runs on the side stream, then the edge rows),
    bit for bit the undivided run.  8 slabs of 40 rows have 5 own rows each,
    fewer than the two edges' 3 + 3 or 4 + 4."""
    from fluidity_b200.slab import NativeSlabs, SlabLayout
    T = 8
    u0, want, rt = _undivided(dtype, shape, T)
    layouts = [SlabLayout(shape, world, r) for r in range(world)]
    ns = NativeSlabs.local(layouts, dtype=dtype)
    a = [u0[:, L.global_slice()].contiguous() for L in layouts]
    b = [ns.new_state(i) for i in range(world)]
    ns.begin(a, b, 0.8, 1.0 / shape[0], 1e30, T)
    ns.steps(T)
    for i in range(world):
        its, rts, done = ns.status(i)
        assert its == T and done and rts == rt
    assert np.array_equal(_gather(layouts, a, want), want)
    ns.close()


def test_native_slab_steps_capture_in_a_graph(cuda):
    """Two eager steps, then two decomposed steps captured once in a CUDA
    graph and replayed three times: the eight-step run."""
    import torch
    from fluidity_b200.slab import NativeSlabs, SlabLayout
    shape, world, T = (64, 48), 2, 8
    u0, want, rt = _undivided("f64", shape, T)
    layouts = [SlabLayout(shape, world, r) for r in range(world)]
    ns = NativeSlabs.local(layouts, dtype="f64")
    a = [u0[:, L.global_slice()].contiguous() for L in layouts]
    b = [ns.new_state(i) for i in range(world)]
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        ns.begin(a, b, 0.8, 1.0 / shape[0], 1e30, T)
        ns.steps(2)   # eager steps first: one-time set-up stays out of the capture
    s.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        ns.steps(2)
    for _ in range(T // 2 - 1):
        g.replay()
    torch.cuda.synchronize()
    its, rts, done = ns.status(0)
    assert its == T and rts == rt
    assert np.array_equal(_gather(layouts, a, want), want)
    del g
    ns.close()


def test_native_slab_nccl_one_rank(cuda):
    """The NCCL transport on one GPU: a communicator of one rank (made from
    an id of fl_slab_nccl_id) and its 64-bit MAX all-reduce each step; no
    neighbours, so no exchange.  Equals the undivided run."""
    from fluidity_b200 import capi
    from fluidity_b200.slab import NativeSlabs, SlabLayout
    if not capi.load().fl_slab_nccl_available():
        pytest.skip("libnccl.so.2 not loadable")
    shape, T = (64, 48), 6
    u0, want, rt = _undivided("f64", shape, T)
    L = SlabLayout(shape, 1, 0)
    ns = NativeSlabs.nccl(L, dtype="f64")
    a = [u0.clone()]
    b = [ns.new_state()]
    ns.begin(a, b, 0.8, 1.0 / shape[0], 1e30, T)
    ns.steps(T)
    its, rts, done = ns.status()
    assert its == T and rts == rt
    assert np.array_equal(a[0].cpu().numpy(), want)
    ns.close()


def test_native_slab_rejects_thin_ghosts(cuda):
    """A slab with a neighbour needs 4 ghost rows on that side."""
    import ctypes as C
    from fluidity_b200 import capi
    lib = capi.load()
    g = capi.Grid.make((32, 40))
    h = C.c_void_p()
    idbuf = (C.c_char * 128)()   # never used: the check comes first
    assert lib.fl_slab_create_nccl(C.byref(h), C.byref(g), 1.4, 0, 0, 3, 40, idbuf, 2, 1) \
        == capi.FL_EINVAL
    assert b"ghost rows" in lib.fl_last_error_string()


@pytest.mark.parametrize("impl", ["native", "python"])
def test_bench_slab_path_one_rank(cuda, capsys, impl):
    """bench.py's multi-GPU path (run_slabs) on one rank and a small grid:
    the native slab step with a one-rank NCCL communicator, or the Python
    schedule, prints a complete line."""
    import argparse
    import json
    import bench
    a = argparse.Namespace(size=64, time_steps=4, dtype="f64", flux="hllc", warmup=3, steps=2,
                           gpus=1, slab_impl=impl, impl="ours")
    bench.run_slabs(a, 1, 0, 0)
    line = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    assert line["value"] > 0 and line["n_gpus"] == 1
    want = "fl_slab_steps (NCCL)" if impl == "native" else "Python schedule over fl_sim_sweep"
    assert line["config"]["slab_step"] == want
