"""Correctness diagnostics of split-solver results: conservation residuals of
one sweep and L1 distances between states.

Conservation.  A sweep updates every cell as U_i + dtdh (F(i-1/2) - F(i+1/2))
with one flux per face (solver/split_solver.hpp:160), so the face fluxes
telescope along each line and

    sum_i U_out - sum_i U_in = dtdh * sum_lines (F(-1/2) - F(N-1/2)).

At a transmissive end the ghost cells mirror the boundary cells
(ghost[-1-g] = cell[g], solver/boundary_loader.hpp:175-199), so both limited
slopes at the boundary face are zero (one one-sided difference is exactly 0),
both evolved states equal the boundary cell's state U_b, and the face flux is
the Riemann flux of (U_b, U_b): the physical flux F(U_b) up to rounding.  The
residual of that identity measures how far a sweep is from conserving mass,
momentum and energy; it is round-off for a conservative kernel.

Everything here runs in float64 on the state's device (torch tensors); the
states are the SoA buffers of the C ABI, shape (dims + 2, pitch).
"""
from __future__ import annotations

import numpy as np
import torch

COMPONENTS = {2: ("rho", "E", "m_x", "m_y"), 3: ("rho", "E", "m_x", "m_y", "m_z"),
              1: ("rho", "E", "m_x")}


def _grid_view(u: torch.Tensor, shape) -> torch.Tensor:
    """(NC, nz, ny, nx) float64 view of the cells of a SoA state."""
    cells = int(np.prod(shape))
    full = tuple(reversed(tuple(shape))) if len(shape) > 1 else (int(shape[0]),)
    return u[:, :cells].to(torch.float64).reshape((u.shape[0],) + full)


def physical_flux(u: torch.Tensor, dim: int, gamma: float) -> torch.Tensor:
    """Conservative flux in dimension dim of states u (NC, ...), float64:
    [m_d, u_d (E + p), m_t u_d (+ p for t = d)] with the state pressure
    p = (gamma - 1)(E - rho |v|^2 / 2) (state/state_impl.hpp:117-128,
    228-244, 293-310)."""
    D = u.shape[0] - 2
    rho, e = u[0], u[1]
    vel = [u[2 + d] / rho for d in range(D)]
    ke = sum(v * v for v in vel)
    p = (gamma - 1.0) * (e - 0.5 * rho * ke)
    vd = vel[dim]
    f = torch.empty_like(u)
    f[0] = u[2 + dim]
    f[1] = vd * (e + p)
    for t in range(D):
        f[2 + t] = u[2 + t] * vd + (p if t == dim else 0.0)
    return f


def sweep_conservation_residual(shape, u_in: torch.Tensor, u_out: torch.Tensor, dim: int,
                                dtdh: float, gamma: float) -> dict:
    """Per component: |sum U_out - sum U_in - dtdh (inflow - outflow)| over
    sum |U_in| + dtdh sum |boundary fluxes|, for one sweep in dim with
    transmissive ends.  Returns {component: relative residual}."""
    D = len(shape)
    a = _grid_view(u_in, shape)
    b = _grid_view(u_out, shape)
    axis = D - dim                           # (NC, z, y, x): x is the last axis
    lo = physical_flux(a.select(axis, 0), dim, gamma)
    hi = physical_flux(a.select(axis, a.shape[axis] - 1), dim, gamma)
    red = tuple(range(1, a.dim()))
    lo, hi = lo.reshape(lo.shape[0], -1), hi.reshape(hi.shape[0], -1)   # (NC, boundary cells)
    d_sum = b.sum(dim=red) - a.sum(dim=red)
    expect = dtdh * (lo.sum(dim=1) - hi.sum(dim=1))
    scale = a.abs().sum(dim=red) + dtdh * (lo.abs().sum(dim=1) + hi.abs().sum(dim=1))
    res = ((d_sum - expect).abs() / scale).cpu().numpy()
    return {name: float(r) for name, r in zip(COMPONENTS[D], res)}


def l1_relative(a: torch.Tensor, b: torch.Tensor, shape) -> dict:
    """Per component sum |a - b| / sum |b| over the cells (b the yardstick)."""
    x = _grid_view(a, shape).flatten(1)
    y = _grid_view(b, shape).flatten(1)
    r = ((x - y).abs().sum(dim=1) / y.abs().sum(dim=1)).cpu().numpy()
    return {name: float(v) for name, v in zip(COMPONENTS[len(shape)], r)}
