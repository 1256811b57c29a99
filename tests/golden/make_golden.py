"""Generates the golden fixtures of tests/golden/ from the reference itself.

Every output array is computed by the reference's own numerics functors
(robclu/fluidity FaceFlux / MHReconstructor / VanLeer / Superbee / Hllc / Force
/ LaxFriedrichs / Richtmyer / State / IdealGas / BoundarySetter and
sim::Parameters), compiled by oracle/build_ref.sh into
oracle/_ref/libfluidity_ref.so and driven by oracle/ref_driver.cpp.  Inputs
are seeded.  Run from the repository root (needs the reference tree to build
the library):

    python oracle/build_ref.sh && python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

from oracle import oracle as O  # noqa: E402
from fluidity_b200.workloads import riemann_states  # noqa: E402
from _util import random_prim  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))
GAMMA = 1.4


def sweep_cases():
    cases = {}
    specs = [
        ("rand1d_64", (64,), [("hllc", "vanleer", "muscl", 0), ("force", "superbee", "muscl", 1),
                              ("lf", "vanleer", "muscl", 0), ("richtmyer", "vanleer", "basic", 1)]),
        ("rand2d_24x20", (24, 20), [("hllc", "vanleer", "muscl", 0), ("force", "vanleer", "muscl", 3),
                                    ("hllc", "superbee", "muscl", 2)]),
        ("smooth2d_32x16", (32, 16), [("hllc", "vanleer", "muscl", 0), ("force", "vanleer", "muscl", 0)]),
        ("rand3d_10x8x6", (10, 8, 6), [("hllc", "vanleer", "muscl", 0), ("force", "superbee", "muscl", 5)]),
    ]
    for seed, (name, shape, pols) in enumerate(specs):
        smooth = name.startswith("smooth")
        u = O.prim_to_cons(random_prim(shape, 100 + seed, smooth=smooth), GAMMA)
        ws = O.ref_max_wavespeed(shape, u, GAMMA)
        dtdh = 0.8 / ws
        for k, (flux, lim, recon, refl) in enumerate(pols):
            for dim in range(len(shape)):
                out = O.ref_sweep(shape, dim, u, GAMMA, dtdh, flux=flux, limiter=lim,
                                  recon=recon, reflect=refl)
                cases[f"{name}__{flux}_{lim}_{recon}_r{refl}_d{dim}"] = dict(
                    shape=np.array(shape), dim=dim, u=u, out=out, dtdh=dtdh, flux=flux,
                    limiter=lim, recon=recon, reflect=refl)
        cases[f"{name}__maxws"] = dict(shape=np.array(shape), u=u, ws=ws)
    return cases


def simulate_cases():
    cases = {}
    # 1-D tube, N = 400, run to t = 0.25 / max initial wavespeed, CFL 0.9
    for seed in (0, 1):
        shape = (400,)
        st = riemann_states(seed, 1)
        u = O.fill_riemann(shape, st, GAMMA)
        t_end = 0.25 / O.ref_max_wavespeed(shape, u, GAMMA)
        out, steps, rt, dts = O.ref_simulate(shape, u, GAMMA, 0.9, 1.0 / 400, t_end, 10 ** 9)
        cases[f"tube1d_400_s{seed}"] = dict(shape=np.array(shape), states=st, u=u, out=out,
                                            steps=steps, run_time=rt, dts=dts, cfl=0.9,
                                            res=1.0 / 400, sim_time=t_end, max_iters=10 ** 9,
                                            flux="hllc", limiter="vanleer", recon="muscl",
                                            reflect=0)
    # 2-D quadrants, 48 x 40, 6 steps, CFL 0.8, HLLC and FORCE
    for flux in ("hllc", "force"):
        shape = (48, 40)
        st = riemann_states(11, 2)
        u = O.fill_riemann(shape, st, GAMMA)
        out, steps, rt, dts = O.ref_simulate(shape, u, GAMMA, 0.8, 1.0 / 48, 1e30, 6, flux=flux)
        cases[f"quad2d_48x40_{flux}"] = dict(shape=np.array(shape), states=st, u=u, out=out,
                                             steps=steps, run_time=rt, dts=dts, cfl=0.8,
                                             res=1.0 / 48, sim_time=1e30, max_iters=6,
                                             flux=flux, limiter="vanleer", recon="muscl",
                                             reflect=0)
    # 3-D octants, 12^3, 3 steps, reflective in all dims
    shape = (12, 12, 12)
    st = riemann_states(22, 3)
    u = O.fill_riemann(shape, st, GAMMA)
    out, steps, rt, dts = O.ref_simulate(shape, u, GAMMA, 0.8, 1.0 / 12, 1e30, 3, reflect=7)
    cases["oct3d_12_reflect"] = dict(shape=np.array(shape), states=st, u=u, out=out, steps=steps,
                                     run_time=rt, dts=dts, cfl=0.8, res=1.0 / 12, sim_time=1e30,
                                     max_iters=3, flux="hllc", limiter="vanleer", recon="muscl",
                                     reflect=7)
    return cases


def check_finite(cases):
    # multi-step cases must stay finite: a blown-up state (NaN) is flagged as
    # an error by the GPU path, while the reference's max_element silently
    # skips NaN wavespeeds, so such runs are not comparable step by step.
    for key, d in cases.items():
        assert np.isfinite(d["out"]).all(), key


def save(name, cases):
    flat = {}
    for key, d in cases.items():
        for k, v in d.items():
            flat[f"{key}::{k}"] = np.asarray(v)
    np.savez_compressed(os.path.join(OUT, name), **flat)


def load(name):
    """Returns {case: {field: value}} from a fixture file."""
    z = np.load(os.path.join(OUT, name), allow_pickle=False)
    cases = {}
    for k in z.files:
        case, field = k.split("::")
        v = z[k]
        cases.setdefault(case, {})[field] = v.item() if v.ndim == 0 else v
    return cases


if __name__ == "__main__":
    if not O.ref_available():
        sys.exit("oracle/_ref/libfluidity_ref.so missing: run oracle/build_ref.sh first")
    save("sweeps.npz", sweep_cases())
    sims = simulate_cases()
    check_finite(sims)
    save("simulate.npz", sims)
    for f in ("sweeps.npz", "simulate.npz"):
        print(f, os.path.getsize(os.path.join(OUT, f)), "bytes")
