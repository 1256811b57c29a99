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
