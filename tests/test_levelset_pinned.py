"""The level-set oracle (oracle/fl_levelset_oracle.c) pinned bit for bit to the
reference's own level-set functors, through tests/golden/levelset.npz
(made by tests/golden/make_golden.py from oracle/ref_driver_ls.cpp):

* HJWeno5 one-sided derivatives (scheme/stencils/weno_hj_5.hpp:51-144);
* GodunovUpwind::forward / backward (scheme/schemes/godunov_upwind.hpp:94-166);
* LevelsetHamiltonian::evaluate (scheme/evaluators/levelset_hamiltonian.hpp:63-98);
* RungeKutta3::update_impl, first and second stage
  (scheme/updaters/runge_kutta_3.hpp:110-148);
* GodunovUpwindScheme::solve, the fast iterative method's local solve
  (scheme/schemes/godunov_upwind_scheme.hpp:37-79);
* the cell body of set_velocities (levelset/cuda/velocity_initialization.cuh:108-143);
* the per-source body of RiemannGFM::invoke: interface normal, the 2-D
  math::interp probes, the rotation into the normal, the two-material HLLC
  star state and the rotation back (ghost_fluid/riemann_ghost_fluid.hpp:70-190).

The CUDA level-set kernels are held to this oracle (tests/test_levelset.py:
velocities and projection bit for bit, the RK3 advection to 1e-12 of max
|phi|), so they are pinned to the reference through it.
Where the reference-functor library is present (it is built from the
reference's sources), the same comparisons also run on fresh seeded fields.
"""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
from make_golden import load  # noqa: E402

ALL = load("levelset.npz")
CASES = {k: v for k, v in ALL.items() if not k.startswith("gfm_")}
GFM = {k: v for k, v in ALL.items() if k.startswith("gfm_")}


@pytest.mark.parametrize("name", sorted(CASES))
def test_levelset_pieces_match_reference_golden(oracle, name):
    c = CASES[name]
    nx, ny, h = int(c["nx"]), int(c["ny"]), float(c["h"])
    back, fwrd = oracle.ls_weno(nx, ny, c["phi"], h)
    assert np.array_equal(back, c["back"]) and np.array_equal(fwrd, c["fwrd"])
    gf, gb = oracle.ls_godunov(nx, ny, c["phi"], h)
    assert np.array_equal(gf, c["god_fwd"]) and np.array_equal(gb, c["god_bwd"])
    assert np.array_equal(oracle.ls_hamiltonian(nx, ny, c["phi"], c["vel"], h), c["ham"])
    s1, s2 = oracle.ls_rk3_stages(nx, ny, c["phi"], c["vel"], float(c["dt"]), h)
    assert np.array_equal(s1, c["stage1"])
    assert np.array_equal(s2, c["stage2"])
    assert np.array_equal(oracle.ls_local_solve(nx, ny, c["band"], h), c["local_band"])
    assert np.array_equal(oracle.ls_local_solve(nx, ny, c["noisy"], h), c["local_noisy"])
    v = oracle.ls_velocity(nx, ny, [c["phi"], -c["phi"]], [c["state0"], c["state1"]], h)
    assert np.array_equal(v, c["velocity"])


@pytest.mark.parametrize("name", sorted(GFM))
def test_gfm_star_states_match_reference_golden(oracle, name):
    """Every source cell of a circular interface: the oracle's GFM star state
    and target cell against the reference's per-source body of
    RiemannGFM::invoke (ghost_fluid/riemann_ghost_fluid.hpp:70-190), bit for
    bit; the reference's 2-D probe interpolation included."""
    c = GFM[name]
    stars, tx, ty = oracle.gfm_star(int(c["nx"]), int(c["ny"]), float(c["h"]), c["ua"], c["ub"],
                                    c["pa"], -c["pa"], (c["ga"], c["gb"]), (c["ia"], c["ib"]),
                                    c["xs"], c["ys"])
    src = np.isfinite(stars[0])
    assert src.sum() == src.size > 20
    assert np.array_equal(stars, c["stars"])
    assert np.array_equal(tx, c["tx"]) and np.array_equal(ty, c["ty"])


def test_goldens_exercise_both_branches():
    """The fixtures reach every branch the pin is about: both signs of the
    velocity (Godunov forward and backward), both cases of the local solve
    (one-sided min + h and the two-sided root), out-of-domain +max
    neighbours, and cells inside and outside each material."""
    both, two_sided, one_sided = False, False, False
    for c in CASES.values():
        both |= bool((c["vel"] > 0).any() and (c["vel"] < 0).any())
        h = float(c["h"])
        d = c["local_band"]
        fin = d[d < 1e300]
        two_sided |= bool((np.abs(fin - np.round(fin / h) * h) > 1e-12 * h).any())
        one_sided |= bool(fin.size)
    assert both and two_sided and one_sided


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_levelset_pieces_match_reference_library(oracle, seed):
    if not oracle.ref_available():
        pytest.skip("reference-functor library not built here (pinned through the goldens)")
    rng = np.random.default_rng(seed)
    nx, ny = int(rng.integers(4, 40)), int(rng.integers(4, 40))
    h = 1.0 / max(nx, ny)
    x = (np.arange(nx) + 0.5) * h
    y = (np.arange(ny) + 0.5) * h
    X, Y = np.meshgrid(x, y)
    c0 = rng.uniform(0.2, 0.8, 2)
    phi = (np.sqrt((X - c0[0]) ** 2 + (Y - c0[1]) ** 2) - rng.uniform(0.1, 0.3)
           + 0.02 * np.sin(7 * X * Y)).ravel()
    vel = rng.uniform(-1.0, 1.0, nx * ny)
    for ref, got in zip(oracle.ls_weno(nx, ny, phi, h, ref=True), oracle.ls_weno(nx, ny, phi, h)):
        assert np.array_equal(ref, got)
    ham = oracle.ls_hamiltonian(nx, ny, phi, vel, h, ref=True)
    assert np.array_equal(oracle.ls_hamiltonian(nx, ny, phi, vel, h), ham)
    dt = 0.3 * h
    s1, s2 = oracle.ls_rk3_stages(nx, ny, phi, vel, dt, h)
    assert np.array_equal(s1, phi - dt * ham)
    assert np.array_equal(s2, oracle.ref_ls_rk3_stage2(nx, ny, phi, s1, vel, dt, h))
    d = np.where(np.abs(phi) < 2 * h, np.abs(phi), np.finfo(np.float64).max)
    assert np.array_equal(oracle.ls_local_solve(nx, ny, d, h),
                          oracle.ls_local_solve(nx, ny, d, h, ref=True))
