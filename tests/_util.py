"""Shared helpers of the test suite: seeded states and the parity metric."""
import numpy as np

from fluidity_b200.workloads import SplitMix64


def random_prim(shape, seed, smooth=False, mild=False):
    """Primitive states with the workloads' value ranges (rho log-uniform in
    [0.1, 10], velocities uniform in [-2, 2], p log-uniform in [0.01, 1000]).
    smooth=True gives a band-limited field instead of white noise; mild=True
    narrows the ranges (rho in [0.5, 2], p in [0.5, 5], |v| <= 0.5) so that
    small grids stay free of the negative pressures MUSCL-Hancock produces
    across five-decade jumps."""
    rng = np.random.default_rng(seed)
    D = len(shape)
    n = int(np.prod(shape))
    prim = np.zeros((D + 2, n))
    if smooth:
        grids = np.meshgrid(*[np.linspace(0, 1, s, endpoint=False) for s in shape[::-1]],
                            indexing="ij")
        x = [g.reshape(-1) for g in grids[::-1]]
        def field(lo, hi):
            f = np.zeros(n)
            for k in range(3):
                ph = rng.uniform(0, 2 * np.pi, D)
                f += sum(np.sin(2 * np.pi * (k + 1) * x[d] + ph[d]) for d in range(D))
            f = (f - f.min()) / (np.ptp(f) + 1e-30)
            return lo + (hi - lo) * f
        rlo, rhi, plo, phi, vmax = (0.5, 2.0, 0.5, 5.0, 0.5) if mild else \
            (0.1, 10.0, 0.01, 1000.0, 2.0)
        prim[0] = np.exp(field(np.log(rlo), np.log(rhi)))
        prim[1] = np.exp(field(np.log(plo), np.log(phi)))
        for d in range(D):
            prim[2 + d] = field(-vmax, vmax)
    else:
        prim[0] = np.exp(rng.uniform(np.log(0.1), np.log(10), n))
        prim[1] = np.exp(rng.uniform(np.log(0.01), np.log(1000), n))
        prim[2:] = rng.uniform(-2, 2, (D, n))
    return prim


def rel_err(a, b, floor_frac=1e-3):
    """Per-cell relative error max_{c,i} |a-b| / max(|b|, floor_frac * max_i |b_c|).
    The floor keeps near-zero momenta (cancellations of O(p) flux terms) from
    dividing by a value far below their component's scale."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    na, nb = np.isnan(a), np.isnan(b)
    if (na != nb).any():
        return float("inf")            # NaN in one result only
    a = np.where(na, 0.0, a)
    b = np.where(nb, 0.0, b)
    scale = np.max(np.abs(b), axis=1, keepdims=True)
    den = np.maximum(np.abs(b), floor_frac * scale)
    den = np.where(den == 0, 1.0, den)
    return float(np.max(np.abs(a - b) / den))
