"""ctypes front end of the CPU oracle and of the reference-functor build.

TEST INFRASTRUCTURE ONLY.  Imported by tests/, ``__graft_entry__.smoke()`` and
bench.py's CPU-baseline leg as the checker; the product never imports it.

* ``liboracle.so`` -- the plain-C restatement (fl_oracle.c) of the reference's
  split-solver arithmetic (FP64 and FP32).
* ``_ref/libfluidity_ref.so`` -- the reference's own functors driven by
  ref_driver.cpp (FP64 only: the reference's MUSCL reconstructor does not
  compile for float, reconstruction/muscl_reconstructor.hpp:112,155).

Arrays are numpy structure-of-arrays with shape ``(D + 2, cells)`` (component
planes ``[rho, E, m_x, m_y, m_z]``, x fastest) unless noted.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libfluidity_ref.so")

FLUX = {"hllc": 0, "force": 1, "lf": 2, "richtmyer": 3}
LIMITER = {"vanleer": 0, "superbee": 1}
RECON = {"muscl": 0, "basic": 1}


class _Grid(C.Structure):
    _fields_ = [("dims", C.c_int32), ("n", C.c_int64 * 3), ("pitch", C.c_int64)]


class _Policy(C.Structure):
    _fields_ = [("flux", C.c_int32), ("limiter", C.c_int32), ("recon", C.c_int32),
                ("flatten", C.c_int32), ("reflect", C.c_uint32)]


def build() -> None:
    """Compile liboracle.so (and, when the reference tree is present, the
    reference-functor library) with the recipes in this folder."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    ref_root = os.environ.get("FLUIDITY_REF", "/root/reference")
    if os.path.isdir(os.path.join(ref_root, "include", "fluidity")):
        subprocess.run(["bash", os.path.join(HERE, "build_ref.sh")], check=True,
                       stdout=subprocess.DEVNULL)


_lib = None
_ref = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            subprocess.run(["make", "-s", "-C", HERE], check=True)
        L = C.CDLL(ORACLE_SO)
        P = C.POINTER
        L.flo_sweep_f64.argtypes = [P(_Grid), C.c_int, C.c_void_p, C.c_void_p,
                                    C.c_double, C.c_double, P(_Policy)]
        L.flo_sweep_f32.argtypes = [P(_Grid), C.c_int, C.c_void_p, C.c_void_p,
                                    C.c_float, C.c_float, P(_Policy)]
        L.flo_max_wavespeed_f64.argtypes = [P(_Grid), C.c_void_p, C.c_double]
        L.flo_max_wavespeed_f64.restype = C.c_double
        L.flo_max_wavespeed_f32.argtypes = [P(_Grid), C.c_void_p, C.c_float]
        L.flo_max_wavespeed_f32.restype = C.c_float
        L.flo_wavespeeds_f64.argtypes = [P(_Grid), C.c_void_p, C.c_double, C.c_void_p]
        L.flo_simulate_f64.argtypes = [P(_Grid), C.c_void_p, C.c_void_p, C.c_double,
                                       C.c_double, C.c_double, C.c_double, C.c_int64,
                                       P(_Policy), P(C.c_int), P(C.c_double), C.c_void_p, C.c_int64]
        L.flo_simulate_f64.restype = C.c_int64
        L.flo_simulate_f32.argtypes = [P(_Grid), C.c_void_p, C.c_void_p, C.c_float,
                                       C.c_float, C.c_double, C.c_float, C.c_int64,
                                       P(_Policy), P(C.c_int), P(C.c_double), C.c_void_p, C.c_int64]
        L.flo_simulate_f32.restype = C.c_int64
        L.flo_prim_to_cons_f64.argtypes = [C.c_int, C.c_void_p, C.c_double, C.c_void_p]
        L.flo_prim_to_cons_f32.argtypes = [C.c_int, C.c_void_p, C.c_float, C.c_void_p]
        L.flo_cons_to_prim_f64.argtypes = [C.c_int, C.c_void_p, C.c_double, C.c_void_p]
        L.flo_flux_f64.argtypes = [C.c_int, C.c_void_p, C.c_double, C.c_int, C.c_void_p]
        L.flo_riemann_f64.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_double,
                                      C.c_double, C.c_int, C.c_int, C.c_void_p]
        L.flo_extend_f64.argtypes = [P(_Grid), C.c_void_p, C.c_int, C.c_uint32, C.c_void_p]
        L.flo_fill_riemann_f64.argtypes = [P(_Grid), C.c_void_p, C.c_double, C.c_void_p]
        L.flo_fill_riemann_f32.argtypes = [P(_Grid), C.c_void_p, C.c_float, C.c_void_p]
        _lib = L
    return _lib


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def ref():
    global _ref
    if _ref is None:
        L = C.CDLL(REF_SO)
        P = C.POINTER
        L.ref_sweep_f64.argtypes = [C.c_int, P(C.c_int64), C.c_int64, C.c_int,
                                    C.c_void_p, C.c_void_p, C.c_double, C.c_double,
                                    C.c_int, C.c_int, C.c_int, C.c_uint32]
        L.ref_max_wavespeed_f64.argtypes = [C.c_int, P(C.c_int64), C.c_int64,
                                            C.c_void_p, C.c_double]
        L.ref_max_wavespeed_f64.restype = C.c_double
        L.ref_simulate_f64.argtypes = [C.c_int, P(C.c_int64), C.c_int64, C.c_void_p,
                                       C.c_void_p, C.c_double, C.c_double, C.c_double,
                                       C.c_double, C.c_int64, C.c_int, C.c_int, C.c_int,
                                       C.c_uint32, P(C.c_int), P(C.c_double), C.c_void_p, C.c_int64]
        L.ref_simulate_f64.restype = C.c_int64
        _ref = L
    return _ref


def _grid(shape) -> _Grid:
    """shape is (nx,), (nx, ny) or (nx, ny, nz) -- x first."""
    g = _Grid()
    g.dims = len(shape)
    n = list(shape) + [1] * (3 - len(shape))
    for d in range(3):
        g.n[d] = int(n[d])
    g.pitch = int(np.prod(shape))
    return g


def _policy(flux="hllc", limiter="vanleer", recon="muscl", flatten=True, reflect=0):
    p = _Policy()
    p.flux = FLUX[flux]
    p.limiter = LIMITER[limiter]
    p.recon = RECON[recon]
    p.flatten = 1 if flatten else 0
    p.reflect = int(reflect)
    return p


def _ptr(a: np.ndarray):
    assert a.flags.c_contiguous
    return a.ctypes.data_as(C.c_void_p)


def sweep(shape, dim, u, gamma, dtdh, **pol):
    """One sweep of the C oracle; u is (D+2, cells) float64 or float32."""
    g = _grid(shape)
    u = np.ascontiguousarray(u)
    out = np.empty_like(u)
    p = _policy(**pol)
    if u.dtype == np.float64:
        rc = lib().flo_sweep_f64(C.byref(g), dim, _ptr(u), _ptr(out), gamma, dtdh, C.byref(p))
    else:
        rc = lib().flo_sweep_f32(C.byref(g), dim, _ptr(u), _ptr(out), gamma, dtdh, C.byref(p))
    if rc != 0:
        raise ValueError(f"oracle sweep failed ({rc})")
    return out


def max_wavespeed(shape, u, gamma):
    g = _grid(shape)
    u = np.ascontiguousarray(u)
    if u.dtype == np.float64:
        return lib().flo_max_wavespeed_f64(C.byref(g), _ptr(u), gamma)
    return np.float32(lib().flo_max_wavespeed_f32(C.byref(g), _ptr(u), gamma))


def wavespeeds(shape, u, gamma):
    g = _grid(shape)
    u = np.ascontiguousarray(u, dtype=np.float64)
    ws = np.empty(u.shape[1], dtype=np.float64)
    lib().flo_wavespeeds_f64(C.byref(g), _ptr(u), gamma, _ptr(ws))
    return ws


def simulate(shape, u, gamma, cfl, res, sim_time, max_iters, **pol):
    """Time loop; returns (state, steps, run_time, dts)."""
    g = _grid(shape)
    a = np.ascontiguousarray(u).copy()
    b = np.empty_like(a)
    in_b = C.c_int(0)
    rt = C.c_double(0)
    cap = int(min(max(int(max_iters), 1), 1 << 20))
    dts = np.zeros(cap, dtype=np.float64)
    p = _policy(**pol)
    f = lib().flo_simulate_f64 if a.dtype == np.float64 else lib().flo_simulate_f32
    steps = f(C.byref(g), _ptr(a), _ptr(b), gamma, cfl, res, sim_time, int(max_iters),
              C.byref(p), C.byref(in_b), C.byref(rt), _ptr(dts), cap)
    if steps < 0:
        raise ValueError("oracle simulate failed")
    return (b if in_b.value else a), int(steps), rt.value, dts[:min(steps, cap)]


def fill_riemann(shape, states_prim, gamma, dtype=np.float64):
    """Piecewise-constant quadrant/octant initial condition (conservative SoA).
    states_prim: (2**D, D+2) primitive states (rho, p, v...)."""
    g = _grid(shape)
    D = len(shape)
    sp = np.ascontiguousarray(states_prim, dtype=dtype).reshape(2 ** D, D + 2)
    out = np.empty((D + 2, int(np.prod(shape))), dtype=dtype)
    if dtype == np.float64:
        lib().flo_fill_riemann_f64(C.byref(g), _ptr(sp), gamma, _ptr(out))
    else:
        lib().flo_fill_riemann_f32(C.byref(g), _ptr(sp), gamma, _ptr(out))
    return out


def prim_to_cons(prim, gamma, dtype=np.float64):
    """Primitive (rho, p, v...) -> conservative; prim is (D+2,) or (D+2, n)."""
    prim = np.asarray(prim, dtype=dtype)
    if prim.ndim == 2:
        cols = [prim_to_cons(prim[:, i], gamma, dtype) for i in range(prim.shape[1])]
        return np.ascontiguousarray(np.stack(cols, axis=1))
    prim = np.ascontiguousarray(prim)
    D = prim.shape[0] - 2
    out = np.empty_like(prim)
    if dtype == np.float64:
        lib().flo_prim_to_cons_f64(D, _ptr(prim), gamma, _ptr(out))
    else:
        lib().flo_prim_to_cons_f32(D, _ptr(prim), gamma, _ptr(out))
    return out


def cons_to_prim(cons, gamma):
    """Conservative -> primitive; cons is (D+2,) or (D+2, n)."""
    cons = np.asarray(cons, dtype=np.float64)
    if cons.ndim == 2:
        cols = [cons_to_prim(cons[:, i], gamma) for i in range(cons.shape[1])]
        return np.ascontiguousarray(np.stack(cols, axis=1))
    cons = np.ascontiguousarray(cons)
    out = np.empty_like(cons)
    lib().flo_cons_to_prim_f64(cons.shape[0] - 2, _ptr(cons), gamma, _ptr(out))
    return out


def flux(cons, gamma, dim):
    cons = np.ascontiguousarray(cons, dtype=np.float64)
    out = np.empty_like(cons)
    lib().flo_flux_f64(cons.shape[0] - 2, _ptr(cons), gamma, dim, _ptr(out))
    return out


def riemann(ul, ur, gamma, dtdh, dim, flux="hllc"):
    ul = np.ascontiguousarray(ul, dtype=np.float64)
    ur = np.ascontiguousarray(ur, dtype=np.float64)
    out = np.empty_like(ul)
    lib().flo_riemann_f64(ul.shape[0] - 2, _ptr(ul), _ptr(ur), gamma, dtdh, dim,
                          FLUX[flux], _ptr(out))
    return out


def extend(shape, u, pad, reflect=0):
    """Ghost-extended grid, (D+2, prod(n_d + 2 pad))."""
    g = _grid(shape)
    D = len(shape)
    u = np.ascontiguousarray(u, dtype=np.float64)
    cells = int(np.prod([n + 2 * pad for n in shape]))
    out = np.empty((D + 2, cells), dtype=np.float64)
    lib().flo_extend_f64(C.byref(g), _ptr(u), pad, reflect, _ptr(out))
    return out


# ---- reference functors (FP64) -----------------------------------------

def ref_sweep(shape, dim, u, gamma, dtdh, flux="hllc", limiter="vanleer",
              recon="muscl", reflect=0):
    D = len(shape)
    n = (C.c_int64 * 3)(*(list(shape) + [1] * (3 - D)))
    u = np.ascontiguousarray(u, dtype=np.float64)
    out = np.empty_like(u)
    rc = ref().ref_sweep_f64(D, n, int(np.prod(shape)), dim, _ptr(u), _ptr(out), gamma,
                             dtdh, FLUX[flux], LIMITER[limiter], RECON[recon], reflect)
    if rc != 0:
        raise ValueError(f"reference sweep failed ({rc})")
    return out


def ref_max_wavespeed(shape, u, gamma):
    D = len(shape)
    n = (C.c_int64 * 3)(*(list(shape) + [1] * (3 - D)))
    u = np.ascontiguousarray(u, dtype=np.float64)
    return ref().ref_max_wavespeed_f64(D, n, int(np.prod(shape)), _ptr(u), gamma)


def ref_simulate(shape, u, gamma, cfl, res, sim_time, max_iters, flux="hllc",
                 limiter="vanleer", recon="muscl", reflect=0):
    D = len(shape)
    n = (C.c_int64 * 3)(*(list(shape) + [1] * (3 - D)))
    a = np.ascontiguousarray(u, dtype=np.float64).copy()
    b = np.empty_like(a)
    in_b = C.c_int(0)
    rt = C.c_double(0)
    cap = int(min(max(int(max_iters), 1), 1 << 20))
    dts = np.zeros(cap, dtype=np.float64)
    steps = ref().ref_simulate_f64(D, n, int(np.prod(shape)), _ptr(a), _ptr(b), gamma, cfl,
                                   res, sim_time, int(max_iters), FLUX[flux],
                                   LIMITER[limiter], RECON[recon], reflect,
                                   C.byref(in_b), C.byref(rt), _ptr(dts), cap)
    if steps < 0:
        raise ValueError("reference simulate failed")
    return (b if in_b.value else a), int(steps), rt.value, dts[:min(steps, cap)]
