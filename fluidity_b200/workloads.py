"""Seeded synthetic inputs for the split-solver workloads.

All draws come from one documented generator, splitmix64 (Steele, Lea and
Flood, "Fast splittable pseudorandom number generators", OOPSLA 2014), feeding
uniform doubles ``(x >> 11) * 2**-53``.  The same draws feed the GPU path and
the CPU checker, so both see bit-identical initial data.

Riemann workloads follow the reference's validation set-ups
(validation/1d_toro_case_*_validation.cu, 2d_liska_case_*): piecewise-constant
primitive states split at the domain midpoint, converted to conservative form
by SimulatorImpl::fill_data (simulator/simulator_impl.hpp:294-340).
"""
from __future__ import annotations

import math

import numpy as np

_MASK = (1 << 64) - 1


class SplitMix64:
    """splitmix64 generator with uniform-double output."""

    def __init__(self, seed: int):
        self.state = seed & _MASK

    def next_u64(self) -> int:
        self.state = (self.state + 0x9E3779B97F4A7C15) & _MASK
        z = self.state
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & _MASK
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & _MASK
        return z ^ (z >> 31)

    def uniform(self, lo: float = 0.0, hi: float = 1.0) -> float:
        u = (self.next_u64() >> 11) * (1.0 / 9007199254740992.0)
        return lo + (hi - lo) * u

    def log_uniform(self, lo: float, hi: float) -> float:
        return math.exp(self.uniform(math.log(lo), math.log(hi)))


def riemann_states(seed: int, dims: int) -> np.ndarray:
    """2**dims primitive states (rho, p, v_x, ...), one per orthant, drawn
    with rho log-uniform in [0.1, 10], each velocity uniform in [-2, 2] and p
    log-uniform in [0.01, 1000].  Orthant index = sum_d (x_d >= 0.5) << d.
    Draw order per orthant: rho, velocities x..z, p."""
    rng = SplitMix64(seed)
    out = np.zeros((2 ** dims, dims + 2), dtype=np.float64)
    for s in range(2 ** dims):
        rho = rng.log_uniform(0.1, 10.0)
        vel = [rng.uniform(-2.0, 2.0) for _ in range(dims)]
        p = rng.log_uniform(0.01, 1000.0)
        out[s, 0] = rho
        out[s, 1] = p
        out[s, 2:] = vel
    return out


def cfl_default(dims: int) -> float:
    """CFL numbers of the workloads: 0.9 for the 1-D tube, 0.8 in 2-D/3-D."""
    return 0.9 if dims == 1 else 0.8


def shock_bubble(seed: int, nx: int = 2048, ny: int = 1024, width: float = 2.0):
    """Two-material shock-bubble set-up on [0, width] x [0, width * ny / nx]
    with cell size h = width / nx.

    Material 0: ambient ideal gas, gamma 1.4, rho 1, p 1, at rest, shocked for
    x < 0.1 by a planar shock of Mach M (uniform in [1.2, 3]) moving in +x
    (post-shock state by the Rankine-Hugoniot relations).  Material 1: a
    circular bubble, gamma 1.67, rho uniform in [0.1, 0.2], p 1, at rest; its
    radius is uniform in [0.1, 0.3] and its centre uniform over the positions
    that keep it inside the domain and clear of the shock.  Level sets are
    signed distances at cell centres (negative inside): phi1 = |x - c| - r,
    phi0 = -phi1.  Draw order: M, rho_bubble, r, c_x, c_y.

    Returns a dict with h, gammas, prim states (rho, p, v_x, v_y) and the two
    level sets as float64 arrays of nx * ny (x fastest)."""
    rng = SplitMix64(seed)
    mach = rng.uniform(1.2, 3.0)
    rho_b = rng.uniform(0.1, 0.2)
    r = rng.uniform(0.1, 0.3)
    h = width / nx
    height = h * ny
    r = min(r, 0.45 * height)
    cx = rng.uniform(0.1 + r + 4 * h + 0.05, width - r - 4 * h)
    cy = rng.uniform(r + 4 * h, height - r - 4 * h)
    g0, g1 = 1.4, 1.67
    a1 = math.sqrt(g0 * 1.0 / 1.0)
    m2 = mach * mach
    rho2 = (g0 + 1.0) * m2 / ((g0 - 1.0) * m2 + 2.0)
    p2 = (2.0 * g0 * m2 - (g0 - 1.0)) / (g0 + 1.0)
    u2 = 2.0 / (g0 + 1.0) * a1 * (mach - 1.0 / mach)
    x = (np.arange(nx) + 0.5) * h
    y = (np.arange(ny) + 0.5) * h
    X, Y = np.meshgrid(x, y)
    phi1 = (np.hypot(X - cx, Y - cy) - r).reshape(-1)
    return {
        "h": h, "nx": nx, "ny": ny, "gammas": (g0, g1), "mach": mach, "centre": (cx, cy),
        "radius": r,
        "ambient": np.array([1.0, 1.0, 0.0, 0.0]),
        "shocked": np.array([rho2, p2, u2, 0.0]),
        "bubble": np.array([rho_b, 1.0, 0.0, 0.0]),
        "shock_phi": (X - 0.1).reshape(-1),      # <= 0 behind the shock
        "phi0": -phi1, "phi1": phi1,
    }
