"""The CPU oracle against the reference: known-answer tests taken from the
reference's own host unit tests, and golden fixtures computed by the
reference's functors (tests/golden/make_golden.py)."""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
from make_golden import load  # noqa: E402

GAMMA = 1.4


# ---- known answers from tests/state_tests_host.cpp -----------------------

def test_prim_cons_round_trip(oracle):
    # state_tests_host.cpp:73-110: rho=1, p=2, v=(3,4)
    prim = np.array([1.0, 2.0, 3.0, 4.0])
    cons = oracle.prim_to_cons(prim, GAMMA)
    back = oracle.cons_to_prim(cons, GAMMA)
    assert cons[0] == 1.0
    assert cons[2] / cons[0] == 3.0 and cons[3] / cons[0] == 4.0
    assert back[0] == 1.0 and back[2] == 3.0 and back[3] == 4.0
    assert abs(back[1] - 2.0) < 1e-15            # tolerance of the reference test


def test_cons_prim_round_trip(oracle):
    # state_tests_host.cpp:112-141: rho=1, m=(2, 2.5), E=3
    cons = np.array([1.0, 3.0, 2.0, 2.5])
    prim = oracle.cons_to_prim(cons, GAMMA)
    conv = oracle.prim_to_cons(prim, GAMMA)
    assert conv[0] == 1.0 and conv[2] == 2.0 and conv[3] == 2.5 and conv[1] == 3.0


def test_conservative_flux_identities(oracle):
    # state_tests_host.cpp:143-194: exact hand formulas for the x flux
    rho, vx, vy, E = 1.0, 2.0, 2.5, 3.0
    p = (GAMMA - 1.0) * (E - 0.5 * rho * (vx * vx + vy * vy))
    f = oracle.flux(np.array([rho, E, rho * vx, rho * vy]), GAMMA, 0)
    assert f[0] == rho * vx
    assert f[1] == vx * (E + p)
    assert f[2] == rho * vx * vx + p
    assert f[3] == rho * vx * vy


# ---- known answers from tests/solver_tests_host.cpp ----------------------

@pytest.mark.parametrize("reflect,expected", [
    (0, [3.0, 2.0, 2.0, 3.0, 4.0, 5.0, 5.0, 4.0]),      # :28-63 transmissive
    (1, [-3.0, -2.0, 2.0, 3.0, 4.0, 5.0, -5.0, -4.0]),  # :65-100 reflective
])
def test_boundary_mirror(oracle, reflect, expected):
    # 8 cells, density 1, velocity 0..7; the reference test treats cells 0,1
    # and 6,7 as ghosts of the interior 2..5 (ghost[-1-g] = cell[g]).
    n = 4
    v = np.arange(2.0, 2.0 + n)
    cons = oracle.prim_to_cons(np.vstack([np.ones(n), np.ones(n), v]), GAMMA)
    ext = oracle.extend((n,), cons, 2, reflect)
    assert np.all(ext[0] == 1.0)
    assert list(ext[2] / ext[0]) == expected


# ---- golden fixtures computed by the reference's functors ----------------

SWEEPS = load("sweeps.npz")
SIMS = load("simulate.npz")


@pytest.mark.parametrize("name", sorted(k for k in SWEEPS if "maxws" not in k))
def test_oracle_sweep_golden(oracle, name):
    c = SWEEPS[name]
    shape = tuple(int(v) for v in c["shape"])
    out = oracle.sweep(shape, int(c["dim"]), c["u"], GAMMA, c["dtdh"], flux=c["flux"],
                       limiter=c["limiter"], recon=c["recon"], reflect=int(c["reflect"]))
    assert np.array_equal(out, c["out"], equal_nan=True), \
        "oracle differs from the reference functors"


@pytest.mark.parametrize("name", sorted(k for k in SWEEPS if "maxws" in k))
def test_oracle_max_wavespeed_golden(oracle, name):
    c = SWEEPS[name]
    shape = tuple(int(v) for v in c["shape"])
    assert oracle.max_wavespeed(shape, c["u"], GAMMA) == c["ws"]


@pytest.mark.parametrize("name", sorted(SIMS))
def test_oracle_simulate_golden(oracle, name):
    c = SIMS[name]
    shape = tuple(int(v) for v in c["shape"])
    u0 = oracle.fill_riemann(shape, c["states"], GAMMA)
    assert np.array_equal(u0, c["u"])
    out, steps, rt, dts = oracle.simulate(shape, u0, GAMMA, c["cfl"], c["res"], c["sim_time"],
                                          c["max_iters"], flux=c["flux"], limiter=c["limiter"],
                                          recon=c["recon"], reflect=int(c["reflect"]))
    assert steps == c["steps"]
    assert rt == c["run_time"]
    assert np.array_equal(dts, c["dts"])
    assert np.array_equal(out, c["out"])


def test_oracle_vs_reference_live(oracle):
    """When the reference build is present (it is built from the reference
    tree, so only where that tree exists), cross-check random cases live."""
    if not oracle.ref_available():
        pytest.skip("reference-functor library not built here")
    from _util import random_prim
    for seed, shape in enumerate([(19,), (9, 7), (5, 6, 4)]):
        u = oracle.prim_to_cons(random_prim(shape, 500 + seed), GAMMA)
        for dim in range(len(shape)):
            for flux in ("hllc", "force"):
                a = oracle.sweep(shape, dim, u, GAMMA, 0.002, flux=flux, reflect=1)
                b = oracle.ref_sweep(shape, dim, u, GAMMA, 0.002, flux=flux, reflect=1)
                assert np.array_equal(a, b, equal_nan=True)


def test_oracle_rejects_small_grid(oracle):
    u = np.ones((3, 3))
    with pytest.raises(ValueError):
        oracle.sweep((3,), 0, u, GAMMA, 0.1)


def test_oracle_f32_close_to_f64(oracle):
    from _util import random_prim, rel_err
    shape = (32, 24)
    u = oracle.prim_to_cons(random_prim(shape, 9, smooth=True), GAMMA)
    ws = oracle.max_wavespeed(shape, u, GAMMA)
    a = oracle.sweep(shape, 0, u, GAMMA, 0.8 / ws)
    b = oracle.sweep(shape, 0, u.astype(np.float32), np.float32(GAMMA), np.float32(0.8 / ws))
    assert rel_err(b, a) < 1e-4
