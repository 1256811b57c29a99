"""Finite differences of the split step against its exact directional
derivative, with the branch decisions counted (CPU, oracle only).

The step is piecewise smooth: limiter cases, the flattening test and its
clamps, and HLLC's pressure clamp, wave-speed forms and wave regions switch
where their comparisons cross.  oracle.sweep_trace records those decisions as
one hash per evolved cell and per face, and oracle.branch_flips counts the
entries where two runs differ.  The exact derivative of the frozen-branch
map at u0 is the oracle's sweep in forward-mode dual numbers with the
flattening coefficient differentiated through its ramp
(oracle.rollout_dual(..., chi_diff=True)).  The claim checked here: a
central difference whose two runs take the same branches everywhere agrees
with that exact derivative to its truncation and round-off (1e-6 relative);
the ones that miss by more straddle flips.  Where chi is active the
frozen-chi derivative (the map the adjoint transposes) differs from both by
the chi terms, and the test shows such a case."""
import numpy as np

from _util import random_prim

GAMMA = 1.4


def _pressure_and_dp(u, du):
    rho, e, mx, my = u
    ke = 0.5 * (mx * mx + my * my) / rho
    p = (GAMMA - 1.0) * (e - ke)
    if du is None:
        return p, None
    drho, de, dmx, dmy = du
    dke = (mx * dmx + my * dmy) / rho - ke * drho / rho
    return p, (GAMMA - 1.0) * (de - dke)


def test_same_rollout_has_no_flips(oracle):
    shape = (24, 20)
    u = oracle.prim_to_cons(random_prim(shape, 3, smooth=True, mild=True), GAMMA)
    _, ta = oracle.rollout_trace(shape, u, GAMMA, [0.1, 0.1])
    out, tb = oracle.rollout_trace(shape, u.copy(), GAMMA, [0.1, 0.1])
    assert oracle.branch_flips(ta, tb) == 0
    # the traced sweep computes what the plain one does
    want = u
    for _ in range(2):
        for d in range(2):
            want = oracle.sweep(shape, d, want, GAMMA, 0.1)
    assert np.array_equal(out, want)


def test_central_differences_without_flips_match_the_exact_derivative(oracle):
    shape = (32, 32)
    n = shape[0] * shape[1]
    rng = np.random.default_rng(4)
    w = rng.uniform(0.5, 1.5, n)
    checked, missed_with_flips, chi_gap = 0, 0, 0
    for seed in range(4):
        prim = random_prim(shape, 10 + seed, smooth=True, mild=True)
        u0 = oracle.prim_to_cons(prim, GAMMA)
        dts = [0.5 / float(oracle.max_wavespeed(shape, u0, GAMMA))] * 4   # CFL 0.5, frozen
        v = np.zeros_like(u0)
        v[0] = rng.standard_normal(n)
        v[1] = rng.standard_normal(n)
        u, du = oracle.rollout_dual(shape, u0, v, GAMMA, dts, chi_diff=True)
        _, dp = _pressure_and_dp(u, du)
        exact = float(np.sum(dp * w))
        assert np.isfinite(u).all() and np.isfinite(exact)
        uf, duf = oracle.rollout_dual(shape, u0, v, GAMMA, dts)
        frozen = float(np.sum(_pressure_and_dp(uf, duf)[1] * w))
        for eps in (1e-3, 1e-5, 1e-6, 1e-7):
            up, tp = oracle.rollout_trace(shape, u0 + eps * v, GAMMA, dts)
            um, tm = oracle.rollout_trace(shape, u0 - eps * v, GAMMA, dts)
            pp, _ = _pressure_and_dp(up, None)
            pm, _ = _pressure_and_dp(um, None)
            fd = float(np.sum((pp - pm) * w)) / (2 * eps)
            err = abs(fd - exact) / abs(exact)
            flips = oracle.branch_flips(tp, tm)
            if flips == 0:
                checked += 1
                assert err <= 1e-6, (seed, eps, err)
                chi_gap += abs(fd - frozen) / abs(frozen) > 1e-3
            elif err > 1e-6:
                missed_with_flips += 1
    assert checked >= 3          # the claim was exercised
    assert chi_gap >= 1          # chi was active somewhere, and its terms showed
    print("central differences without flips:", checked, "; misses, all with flips:",
          missed_with_flips, "; frozen chi off by > 1e-3 without flips:", chi_gap)
