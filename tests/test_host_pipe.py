"""Host-to-host simulation streams (fl_host_pipe_*): every job's result
equals a single device-resident run of the same initial state bit for bit,
whatever the overlap of copies and compute."""
import ctypes as C

import numpy as np
import pytest


def test_pipe_argument_checks():
    """Host-side checks that fail before any device call."""
    from fluidity_b200 import capi
    lib = capi.load()
    g = capi.Grid.make((64, 64))
    h = C.c_void_p()
    assert lib.fl_host_pipe_create(None, C.byref(g), 1.4, 0, 0, 3) == capi.FL_EINVAL
    assert lib.fl_host_pipe_create(C.byref(h), C.byref(g), 1.4, 0, 0, 1) == capi.FL_EINVAL
    assert lib.fl_host_pipe_create(C.byref(h), C.byref(g), 1.4, 0, 0, 5) == capi.FL_EINVAL
    bad = capi.Grid.make((2, 64))
    assert lib.fl_host_pipe_create(C.byref(h), C.byref(bad), 1.4, 0, 0, 3) == capi.FL_EINVAL
    assert lib.fl_host_pipe_run(None, 1, None, None, 0.8, 0.1, 1.0, 10, None,
                                None) == capi.FL_EINVAL
    assert lib.fl_host_pipe_destroy(None) == capi.FL_OK


@pytest.mark.gpu
@pytest.mark.parametrize("sets", [2, 3])
@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_pipe_matches_single_runs(cuda, sets, dtype):
    import torch
    from fluidity_b200.solver import HostPipeline, Simulation, SplitSolver
    shape = (192, 160)
    s = SplitSolver(shape, dtype=dtype, flux="hllc")
    jobs = 5
    host_in, host_out, want = [], [], []
    sim = Simulation(s)
    rng = np.random.default_rng(40)
    for k in range(jobs):
        # moderate orthant states: every run stays finite
        st = np.stack([rng.uniform(0.5, 2.0, 4), rng.uniform(0.5, 5.0, 4),
                       rng.uniform(-0.5, 0.5, 4), rng.uniform(-0.5, 0.5, 4)], axis=1)
        a = s.fill_riemann(st)
        b = torch.empty_like(a)
        host_in.append(a.cpu().pin_memory())
        res, it, rt = sim.run(a.clone(), b, 0.8, 1.0 / 192, 1e30, 12)
        want.append((res.cpu(), it, rt))
        host_out.append(torch.empty_like(host_in[-1]).pin_memory())
    pipe = HostPipeline(s, sets=sets)
    got = pipe.run(host_in, host_out, 0.8, 1.0 / 192, 1e30, 12)
    for k in range(jobs):
        assert got[k] == (want[k][1], want[k][2])
        assert torch.equal(host_out[k], want[k][0]), k


@pytest.mark.gpu
def test_pipe_stiffened(cuda, oracle):
    import torch
    from fluidity_b200.solver import HostPipeline, SplitSolver
    s = SplitSolver((200,), gamma=4.4, p_inf=0.613)
    st = np.array([[1.0, 10.0, 0.0], [1.0, 1.0, 0.0]])
    host_in = [s.fill_riemann(st).cpu().pin_memory()]
    host_out = [torch.empty_like(host_in[0]).pin_memory()]
    (it, rt), = HostPipeline(s).run(host_in, host_out, 0.9, 0.005, 0.05, 10 ** 9)
    with oracle.stiffened(0.613):
        u = oracle.fill_riemann((200,), st, 4.4)
        ref, steps, rt_ref, _ = oracle.simulate((200,), u, 4.4, 0.9, 0.005, 0.05, 10 ** 9)
    assert it == steps
    rel = np.abs(host_out[0].numpy() - ref) / np.maximum(np.abs(ref), 1e-3)
    assert rel.max() < 1e-9
