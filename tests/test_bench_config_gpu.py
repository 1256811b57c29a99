"""Parity and conservation at the headline workload's own size.

The bench's seed-0 four-quadrant Riemann problem at 4096^2 (FP64, HLLC and
FORCE, van Leer MUSCL-Hancock with flattening, CFL 0.8, transmissive) is
stepped twice through the C ABI.  Each GPU step starts from the reference's
state of the step before and is compared with the reference's own functors
(oracle/_ref, the reference's FaceFlux / BoundarySetter / Parameters compiled
from its sources; the pinned C oracle where that library is absent) at the
FP64 bar of the suite: 1e-12 relative per cell (tests/_util.rel_err).  The
same at 1024^2 in FP32 against the FP64 reference, at the FP32 bar (1e-5 of
the component's magnitude).

Conservation: every sweep of the bench workload conserves mass, momentum and
energy up to the fluxes through its transmissive ends, to round-off
(fluidity_b200/diagnostics.py states the identity).
"""
import numpy as np
import pytest

from _util import rel_err

pytestmark = pytest.mark.gpu

GAMMA = 1.4
CFL = 0.8
SEED = 0


def _ref_step(oracle, shape, u, flux):
    """One reference time step (CFL dt from u); returns (state, dt)."""
    res = 1.0 / shape[0]
    if oracle.ref_available():
        out, steps, rt, dts = oracle.ref_simulate(shape, u, GAMMA, CFL, res, 1e30, 1, flux=flux)
    else:
        out, steps, rt, dts = oracle.simulate(shape, u, GAMMA, CFL, res, 1e30, 1, flux=flux)
    assert steps == 1
    return out, rt


def _gpu_step(shape, u, dtype, flux):
    import torch
    from fluidity_b200.solver import Simulation, SplitSolver
    s = SplitSolver(shape, dtype=dtype, flux=flux, gamma=GAMMA)
    tdt = torch.float64 if dtype == "f64" else torch.float32
    a = torch.from_numpy(np.ascontiguousarray(u)).to(device="cuda", dtype=tdt)
    b = torch.empty_like(a)
    res, it, rt = Simulation(s).run(a, b, CFL, 1.0 / shape[0], 1e30, 1)
    assert it == 1
    out = res.cpu().numpy().astype(np.float64)
    del a, b, res
    torch.cuda.empty_cache()
    return out, rt


@pytest.mark.parametrize("flux", ["hllc", "force"])
def test_headline_4096_fp64_steps_match_reference(cuda, oracle, flux):
    from fluidity_b200.workloads import riemann_states
    shape = (4096, 4096)
    u = oracle.fill_riemann(shape, riemann_states(SEED, 2), GAMMA)
    for step in range(2):
        ref, dt_ref = _ref_step(oracle, shape, u, flux)
        got, dt_gpu = _gpu_step(shape, u, "f64", flux)
        assert abs(dt_gpu - dt_ref) <= 1e-14 * dt_ref, (step, dt_gpu, dt_ref)
        e = rel_err(got, ref)
        assert e < 1e-12, f"step {step}: rel err {e:.3e}"
        u = ref


@pytest.mark.parametrize("flux", ["hllc", "force"])
def test_1024_fp32_steps_match_fp64_reference(cuda, oracle, flux):
    """FP32 steps from the reference's FP64 states (rounded to float): within
    1e-5 of each component's magnitude of the FP32 restatement (the
    reference's arithmetic in float, which the reference itself does not
    compile), and within 1e-5 relative L1 per component of the FP64
    reference's step."""
    from fluidity_b200.workloads import riemann_states
    shape = (1024, 1024)
    u = oracle.fill_riemann(shape, riemann_states(SEED, 2), GAMMA)
    for step in range(2):
        ref, dt_ref = _ref_step(oracle, shape, u, flux)
        u32 = u.astype(np.float32)
        ora32, steps, _, _ = oracle.simulate(shape, u32, GAMMA, CFL, 1.0 / shape[0], 1e30, 1,
                                             flux=flux)
        assert steps == 1
        got, dt_gpu = _gpu_step(shape, u32, "f32", flux)
        assert abs(dt_gpu - dt_ref) <= 1e-6 * dt_ref, (step, dt_gpu, dt_ref)
        e = rel_err(got, ora32, 1.0)
        assert e < 1e-5, f"step {step}: normwise rel err vs FP32 restatement {e:.3e}"
        l1 = np.sum(np.abs(got - ref), axis=1) / np.sum(np.abs(ref), axis=1)
        assert np.all(l1 < 1e-5), f"step {step}: relative L1 vs FP64 reference {l1}"
        u = ref


@pytest.mark.parametrize("dtype,bar", [("f64", 1e-13), ("f32", 1e-7)])
@pytest.mark.parametrize("shape", [(4096, 4096), (96, 80), (40, 36, 28)])
def test_sweeps_conserve_to_round_off(cuda, shape, dtype, bar):
    """Each sweep of a few steps of the quadrant / octant problem: the change
    of every component's total equals the flux through the transmissive ends
    to round-off (float64 sums of the stored values; FP32 stores round each
    cell once, which averages out over the grid)."""
    import torch
    from fluidity_b200.diagnostics import sweep_conservation_residual
    from fluidity_b200.solver import SplitSolver
    from fluidity_b200.workloads import riemann_states
    D = len(shape)
    s = SplitSolver(shape, dtype=dtype, gamma=GAMMA)
    a = s.fill_riemann(riemann_states(SEED, D))
    b = torch.empty_like(a)
    worst = {}
    for step in range(3):
        dtdh = CFL / s.max_wavespeed(a).item()
        for dim in range(D):
            s.sweep(a, b, dim, dtdh)
            r = sweep_conservation_residual(shape, a, b, dim, dtdh, GAMMA)
            for k, v in r.items():
                worst[k] = max(worst.get(k, 0.0), v)
            a, b = b, a
    assert max(worst.values()) < bar, worst
