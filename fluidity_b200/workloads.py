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
