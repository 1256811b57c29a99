"""The conservation diagnostic on the CPU oracle's sweeps: the oracle (pinned
to the reference's functors) conserves every component up to the flux through
transmissive ends, and a mistake planted in one cell of its output is seen."""
import numpy as np
import pytest
import torch

from fluidity_b200.diagnostics import l1_relative, sweep_conservation_residual
from fluidity_b200.workloads import riemann_states

GAMMA = 1.4


@pytest.mark.parametrize("shape", [(200,), (40, 30), (12, 10, 9)])
@pytest.mark.parametrize("flux", ["hllc", "force"])
def test_oracle_sweeps_conserve(oracle, shape, flux):
    D = len(shape)
    u = oracle.fill_riemann(shape, riemann_states(5, D), GAMMA)
    for _ in range(3):
        dtdh = 0.8 / oracle.max_wavespeed(shape, u, GAMMA)
        for dim in range(D):
            out = oracle.sweep(shape, dim, u, GAMMA, dtdh, flux=flux)
            r = sweep_conservation_residual(shape, torch.from_numpy(u), torch.from_numpy(out),
                                            dim, dtdh, GAMMA)
            assert max(r.values()) < 1e-13, (dim, r)
            u = out


def test_planted_mistake_is_seen(oracle):
    shape = (40, 30)
    u = oracle.fill_riemann(shape, riemann_states(5, 2), GAMMA)
    dtdh = 0.8 / oracle.max_wavespeed(shape, u, GAMMA)
    out = oracle.sweep(shape, 0, u, GAMMA, dtdh)
    out[1, 617] += 1e-10 * np.abs(u[1]).sum()   # one cell's energy off by 1e-10 of the total
    r = sweep_conservation_residual(shape, torch.from_numpy(u), torch.from_numpy(out), 0,
                                    dtdh, GAMMA)
    assert r["E"] > 1e-13 and r["rho"] < 1e-13


def test_l1_relative(oracle):
    shape = (16, 8)
    u = oracle.fill_riemann(shape, riemann_states(1, 2), GAMMA)
    v = u.copy()
    v[0] *= 1.0 + 1e-6
    r = l1_relative(torch.from_numpy(v), torch.from_numpy(u), shape)
    assert abs(r["rho"] - 1e-6) < 1e-12 and r["E"] == 0.0
