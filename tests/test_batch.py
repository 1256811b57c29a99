"""Batched solver (fl_batch_*): argument checks on CPU, and per-problem parity
with the CPU oracle on the GPU."""
import ctypes as C

import numpy as np
import pytest

from _util import rel_err

GAMMA = 1.4


def small_problems(seed=5, n1d=24, n2d=6):
    from fluidity_b200.batch import batched_workload
    # mild sizes so that the oracle checks every problem within seconds
    return batched_workload(seed=seed, n1d=n1d, n2d=n2d, lo1=16, hi1=600, lo2=16, hi2=72)


def test_workload_shape():
    from fluidity_b200.batch import batched_workload
    probs = batched_workload(n1d=3584, n2d=512)
    assert len(probs) == 4096
    n1 = [s[0] for s, _ in probs[:3584]]
    n2 = [s[0] for s, _ in probs[3584:]]
    assert min(n1) >= 64 and max(n1) <= 8192
    assert min(n2) >= 64 and max(n2) <= 512
    assert all(len(s) == 2 and s[0] == s[1] for s, _ in probs[3584:])
    # log-uniform: the median sits near the geometric mean
    assert 400 < np.median(n1) < 1500


def test_batch_create_rejects_bad_descriptors():
    from fluidity_b200 import build, capi
    build.build()
    lib = capi.load()
    d = (capi.BatchDesc * 1)()
    d[0].dims = 1
    d[0].n[0] = 2          # too small
    d[0].pitch = 32
    d[0].res = 0.1
    h = C.c_void_p()
    assert lib.fl_batch_create(C.byref(h), d, 1, GAMMA, 1, 0) == capi.FL_EINVAL
    assert b"4 cells" in lib.fl_last_error_string()
    d[0].n[0] = 20000      # beyond the shared-memory resident limit
    d[0].pitch = 20000
    assert lib.fl_batch_create(C.byref(h), d, 1, GAMMA, 1, 0) == capi.FL_EINVAL
    d[0].n[0] = 100
    d[0].pitch = 128
    assert lib.fl_batch_create(C.byref(h), d, 1, GAMMA, 1 | capi.FL_FLUX_LF, 0) == capi.FL_EINVAL


def oracle_run(oracle, shape, states, dtype, steps, flux="hllc"):
    npdt = np.float64 if dtype == "f64" else np.float32
    u = oracle.fill_riemann(shape, states, GAMMA, dtype=npdt)
    out, it, rt, _ = oracle.simulate(shape, u, npdt(GAMMA), npdt(0.8), 1.0 / shape[0],
                                     npdt(1e30), steps, flux=flux)
    return out, it


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", ["f64", "f32"])
@pytest.mark.parametrize("mode", ["steps", "graph"])
def test_batch_matches_oracle(cuda, oracle, dtype, mode):
    import torch
    from fluidity_b200.batch import Batch
    probs = small_problems()
    b = Batch(probs, dtype=dtype)
    b.fill()
    steps = 12
    b.begin(0.8, 1e30, steps)
    if mode == "steps":
        b.steps(5)
        b.steps(steps - 5)
    else:
        b.capture(steps)
        b.launch()
    it, rt, done, rc = b.status(allow_nan=True)
    torch.cuda.synchronize()
    checked = 0
    for i, (shape, states) in enumerate(probs):
        ref, rit = oracle_run(oracle, shape, states, dtype, steps)
        if not np.isfinite(ref).all():
            continue                      # blown-up problem: the loop stops it early
        assert it[i] == rit == steps, (i, shape)
        got = b.state(i).double().cpu().numpy()
        tol = 1e-10 if dtype == "f64" else 2e-4
        floor = 1e-3 if dtype == "f64" else 1.0
        assert rel_err(got, ref, floor) < tol, (i, shape)
        checked += 1
    assert checked >= len(probs) // 2


@pytest.mark.gpu
def test_batch_autotune_keeps_results(cuda, oracle):
    import torch
    from fluidity_b200.batch import Batch
    probs = small_problems(seed=9)
    b = Batch(probs, dtype="f64")
    b.fill()
    tune = b.autotune(trial_steps=3)
    assert len(tune["threads_1d"]) == 3 and all(t in (64, 128, 256, 512) for t in tune["threads_1d"])
    assert all(r in (16, 32, 64, 128) for r in tune["strip_rows_2d"])
    b.begin(0.8, 1e30, 6)
    b.steps(6)
    it, _, _, _ = b.status(allow_nan=True)
    for i, (shape, states) in enumerate(probs):
        ref, rit = oracle_run(oracle, shape, states, "f64", 6)
        if np.isfinite(ref).all():
            assert rel_err(b.state(i).cpu().numpy(), ref) < 1e-10


@pytest.mark.gpu
def test_batch_sim_time_stop(cuda, oracle):
    """Each problem stops at its own sim_time like the reference's loop."""
    from fluidity_b200.batch import Batch
    probs = small_problems(seed=2, n1d=10, n2d=3)
    b = Batch(probs, dtype="f64")
    b.fill()
    b.begin(0.8, 0.01, 10 ** 6)
    b.steps(400)
    it, rt, done, rc = b.status(allow_nan=True)
    for i, (shape, states) in enumerate(probs):
        u = oracle.fill_riemann(shape, states, GAMMA)
        ref, rit, rrt, _ = oracle.simulate(shape, u, GAMMA, 0.8, 1.0 / shape[0], 0.01, 10 ** 6)
        if np.isfinite(ref).all() and rit < 400:
            assert it[i] == rit
            assert abs(rt[i] - rrt) <= 1e-12 * rrt


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", ["f64", "f32"])
@pytest.mark.parametrize("flux", ["hllc", "force"])
def test_batch_stiffened_fluid_matches_oracle(cuda, oracle, dtype, flux):
    """Every problem of the batch as the stiffened fluid (p_inf = 0.613, the
    bubble of the two-material tests) against the oracle's stiffened loop;
    the filled states and the step count per problem as well."""
    import torch
    from fluidity_b200.batch import Batch
    p_inf = 0.613
    probs = small_problems(seed=13, n1d=12, n2d=4)
    b = Batch(probs, dtype=dtype, flux=flux, p_inf=p_inf)
    b.fill()
    steps = 10
    b.begin(0.8, 1e30, steps)
    b.capture(steps)
    b.launch()
    it, _, _, _ = b.status(allow_nan=True)
    torch.cuda.synchronize()
    npdt = np.float64 if dtype == "f64" else np.float32
    checked = 0
    with oracle.stiffened(p_inf):
        for i, (shape, states) in enumerate(probs):
            u0 = oracle.fill_riemann(shape, states, GAMMA, dtype=npdt)
            ref, rit, _, _ = oracle.simulate(shape, u0, npdt(GAMMA), npdt(0.8), 1.0 / shape[0],
                                             npdt(1e30), steps, flux=flux)
            if not np.isfinite(ref).all():
                continue
            assert it[i] == rit == steps, (i, shape)
            got = b.state(i).double().cpu().numpy()
            tol = 1e-10 if dtype == "f64" else 2e-4
            floor = 1e-3 if dtype == "f64" else 1.0
            assert rel_err(got, ref, floor) < tol, (i, shape)
            checked += 1
    assert checked >= len(probs) // 2
    # the ideal gas on the same data takes other steps
    g = Batch(probs, dtype=dtype, flux=flux)
    g.fill()
    g.begin(0.8, 1e30, steps)
    g.steps(steps)
    torch.cuda.synchronize()
    assert not torch.equal(g.a, b.a)


def test_batch_set_material_checks():
    from fluidity_b200 import build, capi
    build.build()
    lib = capi.load()
    m = capi.Material(GAMMA, 1.0)
    assert lib.fl_batch_set_material(None, C.byref(m)) == capi.FL_EINVAL
    assert lib.fl_adj_set_material(None, C.byref(m)) == capi.FL_EINVAL
