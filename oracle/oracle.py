"""ctypes front end of the CPU oracle and of the reference-functor build.

TEST INFRASTRUCTURE ONLY.  Imported by tests/, ``__graft_entry__.smoke()`` and
bench.py's CPU-baseline leg as the checker; the product never imports it.

* ``liboracle.so`` -- the plain-C restatement (fl_oracle.c) of the reference's
  split-solver arithmetic (FP64 and FP32); ``liboracle_omp.so`` is the same
  sources with OpenMP, for the timed CPU baseline (``threaded()``).
* ``_ref/libfluidity_ref.so`` -- the reference's own functors driven by
  ref_driver.cpp (FP64 only: the reference's MUSCL reconstructor does not
  compile for float, reconstruction/muscl_reconstructor.hpp:112,155).

Arrays are numpy structure-of-arrays with shape ``(D + 2, cells)`` (component
planes ``[rho, E, m_x, m_y, m_z]``, x fastest) unless noted.
"""
from __future__ import annotations

import contextlib
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
ORACLE_OMP_SO = os.path.join(HERE, "liboracle_omp.so")
REF_SO = os.path.join(HERE, "_ref", "libfluidity_ref.so")

FLUX = {"hllc": 0, "force": 1, "lf": 2, "richtmyer": 3}
LIMITER = {"vanleer": 0, "superbee": 1}
RECON = {"muscl": 0, "basic": 1}


class _Grid(C.Structure):
    _fields_ = [("dims", C.c_int32), ("n", C.c_int64 * 3), ("pitch", C.c_int64)]


class _Policy(C.Structure):
    _fields_ = [("flux", C.c_int32), ("limiter", C.c_int32), ("recon", C.c_int32),
                ("flatten", C.c_int32), ("reflect", C.c_uint32)]


def build(ref_root: str | None = None) -> None:
    """Compile liboracle.so and, when a reference checkout is given (argument
    or FLUIDITY_REF) and present, the reference-functor library, with the
    recipes in this folder."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    ref_root = ref_root or os.environ.get("FLUIDITY_REF")
    if ref_root and os.path.isdir(os.path.join(ref_root, "include", "fluidity")):
        subprocess.run(["bash", os.path.join(HERE, "build_ref.sh"), ref_root], check=True,
                       stdout=subprocess.DEVNULL)


_libs: dict = {}
_threaded = False
_ref = None


@contextlib.contextmanager
def threaded():
    """Within the block the oracle runs from liboracle_omp.so: the same
    sources built with -fopenmp, rows and sweep lines shared among threads
    (OMP_NUM_THREADS, default all host cores), every cell computed as in the
    single-threaded build.  Used to time the CPU baseline."""
    global _threaded
    old = _threaded
    _threaded = True
    try:
        yield lib()
    finally:
        _threaded = old


def threads() -> int:
    """Threads the threaded build uses."""
    return int(os.environ.get("OMP_NUM_THREADS", "0") or 0) or (os.cpu_count() or 1)


def lib():
    path = ORACLE_OMP_SO if _threaded else ORACLE_SO
    L = _libs.get(path)
    if L is None:
        if not os.path.exists(path):
            subprocess.run(["make", "-s", "-C", HERE], check=True)
        L = C.CDLL(path)
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
        L.flo_ls_advect_f64.argtypes = [C.c_int64, C.c_int64, C.c_void_p, C.c_void_p, C.c_double,
                                        C.c_double, C.c_void_p]
        L.flo_ls_velocity_f64.argtypes = [C.c_int64, C.c_int64, C.c_int, C.c_void_p, C.c_void_p,
                                          C.c_int64, C.c_double, C.c_void_p]
        L.flo_ls_project_f64.argtypes = [C.c_int64, C.c_void_p, C.c_void_p]
        L.flo_sweep_trace_f64.argtypes = [P(_Grid), C.c_int, C.c_void_p, C.c_void_p,
                                          C.c_double, C.c_double, P(_Policy), C.c_void_p]
        L.flo_sweep_dual.argtypes = [P(_Grid), C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                     C.c_void_p, C.c_double, C.c_double, P(_Policy)]
        L.flo_sweep_dual_chi.argtypes = L.flo_sweep_dual.argtypes
        L.flo_ls_weno_f64.argtypes = [C.c_int64, C.c_int64, C.c_void_p, C.c_double, C.c_void_p,
                                      C.c_void_p]
        L.flo_ls_godunov_f64.argtypes = [C.c_int64, C.c_int64, C.c_void_p, C.c_double,
                                         C.c_void_p, C.c_void_p]
        L.flo_ls_hamiltonian_f64.argtypes = [C.c_int64, C.c_int64, C.c_void_p, C.c_void_p,
                                             C.c_double, C.c_void_p]
        L.flo_ls_rk3_stages_f64.argtypes = [C.c_int64, C.c_int64, C.c_void_p, C.c_void_p,
                                            C.c_double, C.c_double, C.c_void_p, C.c_void_p]
        L.flo_ls_local_solve_f64.argtypes = [C.c_int64, C.c_int64, C.c_void_p, C.c_double,
                                             C.c_void_p]
        L.flo_mm_gfm_star.argtypes = [C.c_int64, C.c_int64, C.c_int64, C.c_double, C.c_void_p,
                                      C.c_void_p, C.c_void_p, C.c_void_p, C.c_double,
                                      C.c_double, C.c_double, C.c_double, C.c_int64,
                                      C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                      C.c_void_p]
        L.flo_ls_reinit_f64.argtypes = [C.c_int64, C.c_int64, C.c_void_p, C.c_double,
                                        C.c_void_p, C.c_int]
        L.flo_ls_reinit_f64.restype = C.c_int
        L.flo_mm_gfm.argtypes = [C.c_int64, C.c_int64, C.c_int64, C.c_double, C.c_double,
                                 C.c_double, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                 C.c_int]
        L.flo_mm_gfm.restype = C.c_int64
        L.flo_mm_gfm_mat.argtypes = [C.c_int64, C.c_int64, C.c_int64, C.c_double, C.c_double,
                                     C.c_double, C.c_double, C.c_double, C.c_void_p,
                                     C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]
        L.flo_mm_gfm_mat.restype = C.c_int64
        L.flo_mm_extrapolate.argtypes = [C.c_int64, C.c_int64, C.c_int64, C.c_double, C.c_void_p,
                                         C.c_void_p, C.c_int, C.c_int]
        L.flo_mm_extrapolate.restype = C.c_int
        L.flo_mm_set_states.argtypes = [C.c_int64, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p,
                                        C.c_double, C.c_int]
        L.flo_mm_star_left.argtypes = [C.c_void_p, C.c_void_p, C.c_double, C.c_double,
                                       C.c_double, C.c_double, C.c_void_p]
        L.flo_mm_set_states_mat.argtypes = [C.c_int64, C.c_int64, C.c_void_p, C.c_void_p,
                                            C.c_void_p, C.c_double, C.c_double, C.c_int]
        L.flo_mm_combine.argtypes = [C.c_int64, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p]
        L.flo_set_p_inf.argtypes = [C.c_double]
        L.flo_get_p_inf.restype = C.c_double
        _libs[path] = L
    return L


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
        L.ref_set_p_inf.argtypes = [C.c_double]
        L.ref_star_left_2d.argtypes = [C.c_void_p, C.c_void_p, C.c_double, C.c_double,
                                       C.c_double, C.c_double, C.c_void_p]
        L.ref_prim_to_cons_f64.argtypes = [C.c_int, C.c_void_p, C.c_double, C.c_void_p]
        L.ref_ls_weno_2d.argtypes = [C.c_int64, C.c_int64, C.c_void_p, C.c_double, C.c_void_p,
                                     C.c_void_p]
        L.ref_ls_godunov_2d.argtypes = [C.c_int64, C.c_int64, C.c_void_p, C.c_double,
                                        C.c_void_p, C.c_void_p]
        L.ref_ls_hamiltonian_2d.argtypes = [C.c_int64, C.c_int64, C.c_void_p, C.c_void_p,
                                            C.c_double, C.c_void_p]
        L.ref_ls_rk3_stage2_2d.argtypes = [C.c_int64, C.c_int64, C.c_void_p, C.c_void_p,
                                           C.c_void_p, C.c_double, C.c_double, C.c_void_p]
        L.ref_ls_local_solve_2d.argtypes = [C.c_int64, C.c_int64, C.c_void_p, C.c_double,
                                            C.c_void_p]
        L.ref_ls_velocity_2d.argtypes = [C.c_int64, C.c_int64, C.c_int, C.c_void_p, C.c_void_p,
                                         C.c_int64, C.c_double, C.c_void_p]
        L.ref_gfm_star_2d.argtypes = [C.c_int64, C.c_int64, C.c_int64, C.c_double, C.c_void_p,
                                      C.c_void_p, C.c_void_p, C.c_double, C.c_double,
                                      C.c_double, C.c_double, C.c_int64, C.c_void_p,
                                      C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        _ref = L
    return _ref


@contextlib.contextmanager
def stiffened(p_inf: float):
    """Within the block, the oracle (and the reference-functor build, when
    present) compute for the stiffened fluid with this p_inf
    (material/stiff_fluid.hpp:38-133) instead of the ideal gas."""
    lib().flo_set_p_inf(float(p_inf))
    if ref_available():
        ref().ref_set_p_inf(float(p_inf))
    try:
        yield
    finally:
        lib().flo_set_p_inf(0.0)
        if ref_available():
            ref().ref_set_p_inf(0.0)


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


def sweep_dual(shape, dim, u, du, gamma, dtdh, chi_diff=False, **pol):
    """One FP64 sweep in forward-mode dual numbers: (sweep(u), derivative of
    the sweep at u along du), with dtdh held constant and the branches of
    the primal run.  The flattening coefficient is taken as a constant (the
    map the adjoint transposes), or with chi_diff differentiated through its
    ramp (the derivative of the sweep itself where chi is active)."""
    g = _grid(shape)
    u = np.ascontiguousarray(u, dtype=np.float64)
    du = np.ascontiguousarray(du, dtype=np.float64)
    out, dout = np.empty_like(u), np.empty_like(u)
    p = _policy(**pol)
    f = lib().flo_sweep_dual_chi if chi_diff else lib().flo_sweep_dual
    rc = f(C.byref(g), dim, _ptr(u), _ptr(du), _ptr(out), _ptr(dout), gamma, dtdh, C.byref(p))
    if rc != 0:
        raise ValueError(f"dual sweep failed ({rc})")
    return out, dout


def sweep_trace(shape, dim, u, gamma, dtdh, **pol):
    """FP64 sweep with its branch trace: (out, trace), trace one uint64 hash
    of the branch decisions per evolved cell and per face (fl_oracle.h)."""
    g = _grid(shape)
    p = _policy(**pol)
    u = np.ascontiguousarray(u, dtype=np.float64)
    out = np.empty_like(u)
    n = shape[dim]
    lines = int(np.prod(shape)) // n
    trace = np.zeros(lines * (2 * n + 3), dtype=np.uint64)
    rc = lib().flo_sweep_trace_f64(C.byref(g), dim, _ptr(u), _ptr(out), gamma, dtdh,
                                   C.byref(p), _ptr(trace))
    if rc != 0:
        raise RuntimeError(f"flo_sweep_trace_f64 failed ({rc})")
    return out, trace


def rollout_trace(shape, u, gamma, dtdh_seq, **pol):
    """Steps with the given dt/dh sequence (sweeps x, y, z each step):
    (final state, one branch trace per sweep)."""
    traces = []
    for dtdh in dtdh_seq:
        for dim in range(len(shape)):
            u, t = sweep_trace(shape, dim, u, gamma, float(dtdh), **pol)
            traces.append(t)
    return u, traces


def branch_flips(traces_a, traces_b) -> int:
    """Entries (evolved cells and faces over all sweeps) whose branch
    decisions differ between two traced rollouts of the same shape."""
    return int(sum(int(np.count_nonzero(a != b)) for a, b in zip(traces_a, traces_b)))


def rollout_dual(shape, u, du, gamma, dtdh_seq, chi_diff=False, **pol):
    """Steps with the given dt/dh sequence (sweeps x, y, z each step), in dual
    numbers: returns the final state and its derivative along du (chi frozen,
    or differentiated with chi_diff)."""
    for dtdh in dtdh_seq:
        for dim in range(len(shape)):
            u, du = sweep_dual(shape, dim, u, du, gamma, float(dtdh), chi_diff=chi_diff, **pol)
    return u, du


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


def ref_prim_to_cons(prim, gamma):
    """The reference's State::conservative of one primitive state (FP64)."""
    prim = np.ascontiguousarray(prim, dtype=np.float64)
    out = np.empty_like(prim)
    ref().ref_prim_to_cons_f64(prim.shape[0] - 2, _ptr(prim), gamma, _ptr(out))
    return out


def mm_star_left(ul, ur, gl, il, gr, ir):
    """The oracle's two-material HLLC star state (left side, normal x)."""
    ul = np.ascontiguousarray(ul, dtype=np.float64)
    ur = np.ascontiguousarray(ur, dtype=np.float64)
    out = np.empty(4)
    lib().flo_mm_star_left(_ptr(ul), _ptr(ur), gl, il, gr, ir, _ptr(out))
    return out


def ref_star_left(ul, ur, gl, il, gr, ir):
    """The reference's Hllc::solve_star_conservative_left, 2-D states."""
    ul = np.ascontiguousarray(ul, dtype=np.float64)
    ur = np.ascontiguousarray(ur, dtype=np.float64)
    out = np.empty(4)
    ref().ref_star_left_2d(_ptr(ul), _ptr(ur), gl, il, gr, ir, _ptr(out))
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


# ---- level set (FP64, 2-D; arrays are (cells,) with x fastest) -------------

def ls_advect(nx, ny, phi, vel, dt, h):
    phi = np.ascontiguousarray(phi, dtype=np.float64)
    vel = np.ascontiguousarray(vel, dtype=np.float64)
    out = np.empty_like(phi)
    lib().flo_ls_advect_f64(nx, ny, _ptr(phi), _ptr(vel), dt, h, _ptr(out))
    return out


def ls_velocity(nx, ny, phis, states, h):
    """phis: list of (cells,) level sets; states: list of (4, pitch) states."""
    phis = [np.ascontiguousarray(p, dtype=np.float64) for p in phis]
    states = [np.ascontiguousarray(s, dtype=np.float64) for s in states]
    pitch = states[0].shape[1]
    pp = (C.c_void_p * len(phis))(*[p.ctypes.data for p in phis])
    sp = (C.c_void_p * len(states))(*[s.ctypes.data for s in states])
    out = np.empty(nx * ny, dtype=np.float64)
    lib().flo_ls_velocity_f64(nx, ny, len(phis), pp, sp, pitch, h, _ptr(out))
    return out


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def ls_weno(nx, ny, phi, h, ref=False):
    """One-sided WENO-HJ5 derivatives (back, fwrd), each (2, cells): the
    oracle's, or with ref=True the reference's HJWeno5 functors."""
    phi = _f64(phi)
    back = np.empty((2, nx * ny))
    fwrd = np.empty((2, nx * ny))
    f = globals()["ref"]().ref_ls_weno_2d if ref else lib().flo_ls_weno_f64
    f(nx, ny, _ptr(phi), h, _ptr(back), _ptr(fwrd))
    return back, fwrd


def ls_godunov(nx, ny, phi, h, ref=False):
    """Godunov upwind |grad phi| for v <= 0 (forward) and v > 0 (backward)."""
    phi = _f64(phi)
    fwd = np.empty(nx * ny)
    bwd = np.empty(nx * ny)
    f = globals()["ref"]().ref_ls_godunov_2d if ref else lib().flo_ls_godunov_f64
    f(nx, ny, _ptr(phi), h, _ptr(fwd), _ptr(bwd))
    return fwd, bwd


def ls_hamiltonian(nx, ny, phi, vel, h, ref=False):
    phi, vel = _f64(phi), _f64(vel)
    out = np.empty(nx * ny)
    f = globals()["ref"]().ref_ls_hamiltonian_2d if ref else lib().flo_ls_hamiltonian_f64
    f(nx, ny, _ptr(phi), _ptr(vel), h, _ptr(out))
    return out


def ls_rk3_stages(nx, ny, phi, vel, dt, h):
    """The oracle's first two RK3 stages (s1, s2)."""
    phi, vel = _f64(phi), _f64(vel)
    s1, s2 = np.empty(nx * ny), np.empty(nx * ny)
    lib().flo_ls_rk3_stages_f64(nx, ny, _ptr(phi), _ptr(vel), dt, h, _ptr(s1), _ptr(s2))
    return s1, s2


def ref_ls_rk3_stage2(nx, ny, phi, stage1, vel, dt, h):
    """The reference's RungeKutta3::update_impl second stage per cell, given
    the first stage over the whole grid."""
    phi, stage1, vel = _f64(phi), _f64(stage1), _f64(vel)
    out = np.empty(nx * ny)
    ref().ref_ls_rk3_stage2_2d(nx, ny, _ptr(phi), _ptr(stage1), _ptr(vel), dt, h, _ptr(out))
    return out


def ls_local_solve(nx, ny, d, h, ref=False):
    d = _f64(d)
    out = np.empty(nx * ny)
    f = globals()["ref"]().ref_ls_local_solve_2d if ref else lib().flo_ls_local_solve_f64
    f(nx, ny, _ptr(d), h, _ptr(out))
    return out


def ref_ls_velocity(nx, ny, phis, states, h):
    """The reference's per-cell set_velocities body (see ls_velocity)."""
    phis = [_f64(p) for p in phis]
    states = [_f64(s) for s in states]
    pitch = states[0].shape[1]
    pp = (C.c_void_p * len(phis))(*[p.ctypes.data for p in phis])
    sp = (C.c_void_p * len(states))(*[s.ctypes.data for s in states])
    out = np.empty(nx * ny, dtype=np.float64)
    ref().ref_ls_velocity_2d(nx, ny, len(phis), pp, sp, pitch, h, _ptr(out))
    return out


def gfm_star(nx, ny, h, ua, ub, pa, pb, gammas, p_infs, xs, ys, ref=False):
    """Star states (4, k) and target offsets (tx, ty) of the GFM for source
    cells (xs, ys) of material A: the oracle's (cells that are not sources
    get NaN), or with ref=True the reference's per-source body."""
    ua, ub, pa = _f64(ua), _f64(ub), _f64(pa)
    pitch = ua.shape[1]
    xs = np.ascontiguousarray(xs, dtype=np.int64)
    ys = np.ascontiguousarray(ys, dtype=np.int64)
    k = xs.size
    stars = np.empty((k, 4))
    tx = np.zeros(k, dtype=np.int32)
    ty = np.zeros(k, dtype=np.int32)
    (ga, gb), (ia, ib) = gammas, p_infs
    if ref:
        globals()["ref"]().ref_gfm_star_2d(nx, ny, pitch, h, _ptr(ua), _ptr(ub), _ptr(pa), ga, ia,
                                           gb, ib, k, _ptr(xs), _ptr(ys), _ptr(stars), _ptr(tx),
                                           _ptr(ty))
    else:
        pb = _f64(pb)
        lib().flo_mm_gfm_star(nx, ny, pitch, h, _ptr(ua), _ptr(ub), _ptr(pa), _ptr(pb), ga, ia,
                              gb, ib, k, _ptr(xs), _ptr(ys), _ptr(stars), _ptr(tx), _ptr(ty))
    return stars.T.copy(), tx, ty


def ls_project(a, b):
    a = np.ascontiguousarray(a, dtype=np.float64).copy()
    b = np.ascontiguousarray(b, dtype=np.float64).copy()
    lib().flo_ls_project_f64(a.size, _ptr(a), _ptr(b))
    return a, b


def ls_reinit(nx, ny, phi, h, max_sweeps=100000):
    phi = np.ascontiguousarray(phi, dtype=np.float64)
    out = np.empty_like(phi)
    sweeps = lib().flo_ls_reinit_f64(nx, ny, _ptr(phi), h, _ptr(out), max_sweeps)
    return out, sweeps


# ---- two-material ghost-fluid path (fl_mm_oracle.c) ---------------------------
# States: (4, pitch) arrays, float64 or float32 (FP32 values are carried as
# doubles in the C code and rounded back to float on every store).

def _as_f64(u):
    return np.ascontiguousarray(u, dtype=np.float64).copy()


def mm_gfm(nx, ny, h, gammas, u0, u1, phi0, phi1, p_infs=(0.0, 0.0)):
    """Riemann ghost-fluid star states for both materials; returns (u0, u1, n).
    p_infs: each material's stiffened-fluid constant (0: ideal gas)."""
    f32 = u0.dtype == np.float32
    a, b = _as_f64(u0), _as_f64(u1)
    p0 = np.ascontiguousarray(phi0, dtype=np.float64)
    p1 = np.ascontiguousarray(phi1, dtype=np.float64)
    n = lib().flo_mm_gfm_mat(nx, ny, a.shape[1], h, gammas[0], p_infs[0], gammas[1], p_infs[1],
                             _ptr(a), _ptr(b), _ptr(p0), _ptr(p1), int(f32))
    dt = np.float32 if f32 else np.float64
    return a.astype(dt), b.astype(dt), int(n)


def mm_extrapolate(nx, ny, h, u, phi, max_iters=64):
    """Ghost-cell extrapolation of one material; returns (u, sweeps)."""
    f32 = u.dtype == np.float32
    a = _as_f64(u)
    p = np.ascontiguousarray(phi, dtype=np.float64)
    it = lib().flo_mm_extrapolate(nx, ny, a.shape[1], h, _ptr(a), _ptr(p), int(f32), max_iters)
    return a.astype(u.dtype), int(it)


def mm_ghost(nx, ny, h, gammas, u0, u1, phi0, phi1, max_iters=64, p_infs=(0.0, 0.0)):
    """GFM for both materials, then the extrapolation of each."""
    u0, u1, _ = mm_gfm(nx, ny, h, gammas, u0, u1, phi0, phi1, p_infs)
    u0, _ = mm_extrapolate(nx, ny, h, u0, phi0, max_iters)
    u1, _ = mm_extrapolate(nx, ny, h, u1, phi1, max_iters)
    return u0, u1


def mm_set_states(u, phi, prim, gamma, p_inf=0.0):
    f32 = u.dtype == np.float32
    a = _as_f64(u)
    p = np.ascontiguousarray(phi, dtype=np.float64)
    pr = np.ascontiguousarray(prim, dtype=np.float64)
    lib().flo_mm_set_states_mat(p.size, a.shape[1], _ptr(a), _ptr(p), _ptr(pr), gamma, p_inf,
                                int(f32))
    return a.astype(u.dtype)


def mm_combine(u0, u1, phi1):
    a = _as_f64(u0)
    b = _as_f64(u1)
    p = np.ascontiguousarray(phi1, dtype=np.float64)
    lib().flo_mm_combine(p.size, a.shape[1], _ptr(a), _ptr(b), _ptr(p))
    return a.astype(u0.dtype)


def mm_step(nx, ny, h, gammas, cfl, u0, u1, phi0, phi1, reinit, max_iters=64,
            p_infs=(0.0, 0.0)):
    """One step of the two-material loop: ghost cells, CFL time step over
    both materials, split MUSCL-Hancock/HLLC step of each material with its
    own equation of state, level-set velocity, RK3 advection, projection and
    (when reinit) reinitialisation of both level sets.  Returns
    (u0, u1, phi0, phi1, dt)."""
    shape = (nx, ny)
    u0, u1 = mm_ghost(nx, ny, h, gammas, u0, u1, phi0, phi1, max_iters, p_infs)
    ws = []
    for u, g, pi in ((u0, gammas[0], p_infs[0]), (u1, gammas[1], p_infs[1])):
        with stiffened(pi):
            ws.append(float(max_wavespeed(shape, u, g)))
    dt = cfl * h / max(ws)
    dtdh = dt / h
    out = []
    for u, g, pi in ((u0, gammas[0], p_infs[0]), (u1, gammas[1], p_infs[1])):
        with stiffened(pi):
            v = sweep(shape, 0, u, g, dtdh)
            v = sweep(shape, 1, v, g, dtdh)
        out.append(v)
    u0, u1 = out
    vel = ls_velocity(nx, ny, [phi0, phi1], [u0.astype(np.float64), u1.astype(np.float64)], h)
    a = ls_advect(nx, ny, phi0, vel, dt, h)
    b = ls_advect(nx, ny, phi1, vel, dt, h)
    a, b = ls_project(a, b)
    if reinit:
        a, _ = ls_reinit(nx, ny, a, h)
        b, _ = ls_reinit(nx, ny, b, h)
    return u0, u1, a, b, dt
