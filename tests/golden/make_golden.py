"""Generates the golden fixtures of tests/golden/ from the reference itself.

Every output array is computed by the reference's own numerics functors
(robclu/fluidity FaceFlux / MHReconstructor / VanLeer / Superbee / Hllc / Force
/ LaxFriedrichs / Richtmyer / State / IdealGas / BoundarySetter and
sim::Parameters), compiled by oracle/build_ref.sh into
oracle/_ref/libfluidity_ref.so and driven by oracle/ref_driver.cpp.  Inputs
are seeded.  Run from the repository root (needs the reference tree to build
the library):

    bash oracle/build_ref.sh REFERENCE_ROOT && python tests/golden/make_golden.py

stiff.npz holds the same kinds of cases for the stiffened fluid.

levelset.npz holds the reference's level-set functors on seeded 2-D fields
(oracle/ref_driver_ls.cpp): HJWeno5 one-sided derivatives, GodunovUpwind
gradients, LevelsetHamiltonian values, the first two RungeKutta3 stages, the
GodunovUpwindScheme local eikonal solve and the set_velocities cell body.
`python tests/golden/make_golden.py levelset` regenerates that file alone.
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


# Stiffened fluid (material/stiff_fluid.hpp:38-133): the reference's
# StiffFluid(gamma, p_inf) in place of IdealGas; (4.4, 0.613) is the water of
# the reference's gas-water validation (StiffFluid{4.4} keeps p_inf = 0.613).
STIFF = [(4.4, 0.613), (6.12, 343.0)]


def stiff_cases():
    cases = {}
    specs = [("rand1d_64", (64,), 0), ("smooth2d_32x16", (32, 16), 3),
             ("rand3d_10x8x6", (10, 8, 6), 5)]
    pols = [("hllc", "vanleer", "muscl"), ("force", "superbee", "muscl"),
            ("lf", "vanleer", "basic"), ("richtmyer", "vanleer", "muscl")]
    for k, (gamma, p_inf) in enumerate(STIFF):
        with O.stiffened(p_inf):
            for seed, (name, shape, refl) in enumerate(specs):
                smooth = name.startswith("smooth")
                prim = random_prim(shape, 300 + 10 * k + seed, smooth=smooth, mild=True)
                u = np.stack([O.ref_prim_to_cons(prim[:, i], gamma)
                              for i in range(prim.shape[1])], axis=1)
                ws = O.ref_max_wavespeed(shape, u, gamma)
                dtdh = 0.8 / ws
                tag = f"g{k}_{name}"
                cases[f"{tag}__maxws"] = dict(shape=np.array(shape), u=u, ws=ws, gamma=gamma,
                                              p_inf=p_inf, prim=prim)
                for flux, lim, recon in pols:
                    for dim in range(len(shape)):
                        out = O.ref_sweep(shape, dim, u, gamma, dtdh, flux=flux, limiter=lim,
                                          recon=recon, reflect=refl)
                        # input: the u of case "<tag>__maxws"
                        cases[f"{tag}__{flux}_{lim}_{recon}_d{dim}"] = dict(
                            shape=np.array(shape), dim=dim, src=tag, out=out, dtdh=dtdh,
                            flux=flux, limiter=lim, recon=recon, reflect=refl, gamma=gamma,
                            p_inf=p_inf)
            # whole runs: a 1-D tube and 2-D quadrants, filled as fill_data does
            for name, shape, dims_seed, cfl, steps, flux in (
                    ("tube1d_200", (200,), 31, 0.9, 40, "hllc"),
                    ("quad2d_40x32", (40, 32), 32, 0.8, 6, "force")):
                D = len(shape)
                st = riemann_states(dims_seed, D)
                u = O.fill_riemann(shape, st, gamma)
                for i in range(2 ** D):       # the oracle's fill against the reference's
                    ref_c = O.ref_prim_to_cons(st[i], gamma)
                    assert np.array_equal(O.prim_to_cons(st[i], gamma), ref_c)
                out, n, rt, dts = O.ref_simulate(shape, u, gamma, cfl, 1.0 / shape[0], 1e30,
                                                 steps, flux=flux)
                cases[f"g{k}_{name}_{flux}"] = dict(
                    shape=np.array(shape), states=st, u=u, out=out, steps=n, run_time=rt,
                    dts=dts, cfl=cfl, res=1.0 / shape[0], sim_time=1e30, max_iters=steps,
                    flux=flux, limiter="vanleer", recon="muscl", reflect=0, gamma=gamma,
                    p_inf=p_inf)
    # the two-material HLLC star state (Hllc::solve_star_conservative_left,
    # flux_hllc.hpp:330-361) for every pairing of ideal gas and stiffened fluid
    rng = np.random.default_rng(77)
    for k in range(64):
        gl, gr = rng.uniform(1.1, 6.0, 2)
        il = 0.0 if k % 4 in (0, 1) else float(rng.uniform(0.0, 50.0))
        ir = 0.0 if k % 4 in (0, 2) else float(rng.uniform(0.0, 50.0))
        sides = []
        for g, pi in ((gl, il), (gr, ir)):
            prim = np.array([rng.uniform(0.5, 3.0), rng.uniform(0.5, 20.0),
                             rng.uniform(-2.0, 2.0), rng.uniform(-2.0, 2.0)])
            with O.stiffened(pi):
                sides.append(O.ref_prim_to_cons(prim, g))
        star = O.ref_star_left(sides[0], sides[1], gl, il, gr, ir)
        cases[f"star_{k:02d}"] = dict(ul=sides[0], ur=sides[1], gl=gl, il=il, gr=gr, ir=ir,
                                      star=star)
    return cases


def levelset_cases():
    cases = {}
    rng = np.random.default_rng(2024)
    big = np.finfo(np.float64).max

    def grid(nx, ny):
        h = 1.0 / ny
        x = (np.arange(nx) + 0.5) * h
        y = (np.arange(ny) + 0.5) * h
        return h, np.meshgrid(x, y)

    specs = []
    h, (X, Y) = grid(40, 32)
    specs.append(("circle_40x32", 40, 32, h, np.sqrt((X - 0.6) ** 2 + (Y - 0.5) ** 2) - 0.3,
                  np.sin(3 * X) * np.cos(2 * Y)))
    h, (X, Y) = grid(36, 28)
    d1 = np.sqrt((X - 0.4) ** 2 + (Y - 0.5) ** 2) - 0.25
    d2 = np.sqrt((X - 0.9) ** 2 + (Y - 0.45) ** 2) - 0.2
    specs.append(("two_circles_36x28", 36, 28, h, np.minimum(d1, d2), -0.5 + X - 0.3 * Y))
    h, (X, Y) = grid(24, 20)
    specs.append(("wavy_24x20", 24, 20, h,
                  0.3 * np.sin(2 * np.pi * X) + 0.2 * np.cos(3 * np.pi * Y) - 0.1,
                  rng.uniform(-1.0, 1.0, (20, 24))))
    h, (X, Y) = grid(4, 40)
    specs.append(("thin_4x40", 4, 40, h, np.sin(5 * Y) - 0.3 + 0.1 * X,
                  rng.uniform(-2.0, 2.0, (40, 4))))
    for name, nx, ny, h, phi, vel in specs:
        phi = np.ascontiguousarray(phi.ravel())
        vel = np.ascontiguousarray(vel.ravel())
        back, fwrd = O.ls_weno(nx, ny, phi, h, ref=True)
        gf, gb = O.ls_godunov(nx, ny, phi, h, ref=True)
        ham = O.ls_hamiltonian(nx, ny, phi, vel, h, ref=True)
        dt = 0.4 * h / np.max(np.abs(vel))
        stage1 = phi - dt * ham                # RungeKutta3::update_impl's first line
        stage2 = O.ref_ls_rk3_stage2(nx, ny, phi, stage1, vel, dt, h)
        # local eikonal solve: a band of distances near the interface (a
        # fast-iterative-method start) and, separately, distances with noise
        band = np.where(np.abs(phi) < 1.5 * h, np.abs(phi), big)
        noisy = np.abs(phi) * (1.0 + 0.05 * rng.standard_normal(phi.size))
        loc_band = O.ls_local_solve(nx, ny, band, h, ref=True)
        loc_noisy = O.ls_local_solve(nx, ny, noisy, h, ref=True)
        states = [np.vstack([rng.uniform(0.5, 2.0, phi.size), rng.uniform(2.0, 8.0, phi.size),
                             rng.uniform(-1.0, 1.0, phi.size), rng.uniform(-1.0, 1.0, phi.size)])
                  for _ in range(2)]
        v = O.ref_ls_velocity(nx, ny, [phi, -phi], states, h)
        cases[name] = dict(nx=nx, ny=ny, h=h, dt=dt, phi=phi, vel=vel, back=back, fwrd=fwrd,
                           god_fwd=gf, god_bwd=gb, ham=ham, stage1=stage1, stage2=stage2,
                           band=band, local_band=loc_band, noisy=noisy, local_noisy=loc_noisy,
                           state0=states[0], state1=states[1], velocity=v)
    # Riemann ghost fluid: star states and targets of every source cell of a
    # circular interface, for ideal-gas and stiffened-fluid pairings
    h, (X, Y) = grid(48, 40)
    pa = (np.sqrt((X - 0.6) ** 2 + (Y - 0.5) ** 2) - 0.3).ravel()

    def smooth_states(g, pinf, k):
        rho = 1.0 + 0.3 * np.sin((5 + k) * X) * np.cos(3 * Y)
        u = 0.3 * np.cos((4 + k) * Y)
        v = 0.2 * np.sin(3 * X + k)
        p = 1.0 + 0.5 * np.cos(2 * X + Y)
        e = (p + g * pinf) / (g - 1.0) + 0.5 * rho * (u * u + v * v)
        return np.vstack([rho.ravel(), e.ravel(), (rho * u).ravel(), (rho * v).ravel()])

    cand = np.nonzero((pa <= 0.0) & (pa >= -h))[0]
    for k, ((ga, gb), (ia, ib)) in enumerate([((1.4, 1.67), (0.0, 0.0)),
                                               ((1.4, 4.4), (0.0, 0.6)),
                                               ((5.5, 1.4), (0.613, 0.0)),
                                               ((4.4, 5.5), (0.3, 0.613))]):
        ua, ub = smooth_states(ga, ia, k), smooth_states(gb, ib, k + 1)
        xs, ys = cand % 48, cand // 48
        stars, tx, ty = O.gfm_star(48, 40, h, ua, ub, pa, -pa, (ga, gb), (ia, ib), xs, ys,
                                   ref=True)
        cases[f"gfm_{k}"] = dict(nx=48, ny=40, h=h, ua=ua, ub=ub, pa=pa, ga=ga, gb=gb, ia=ia,
                                 ib=ib, xs=xs, ys=ys, stars=stars, tx=tx, ty=ty)
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
    if sys.argv[1:] == ["levelset"]:
        save("levelset.npz", levelset_cases())
        print("levelset.npz", os.path.getsize(os.path.join(OUT, "levelset.npz")), "bytes")
        sys.exit(0)
    save("levelset.npz", levelset_cases())
    save("sweeps.npz", sweep_cases())
    sims = simulate_cases()
    check_finite(sims)
    save("simulate.npz", sims)
    stiff = stiff_cases()
    check_finite({k: v for k, v in stiff.items() if "out" in v and "dim" not in v})
    save("stiff.npz", stiff)
    for f in ("sweeps.npz", "simulate.npz", "stiff.npz", "levelset.npz"):
        print(f, os.path.getsize(os.path.join(OUT, f)), "bytes")
