"""ctypes binding of the C ABI declared in include/fluidity_b200.h.

The library is built in-tree (fluidity_b200/libfluidity_b200.so).  Loading
fails loudly when it is missing: there is no fallback implementation.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libfluidity_b200.so")

FL_OK, FL_EINVAL, FL_ECUDA, FL_ETIMEOUT, FL_ENAN, FL_ENOMEM = 0, 1, 2, 3, 4, 5

FL_DTYPE_F64 = 0
FL_DTYPE_F32 = 1
FL_FLUX_HLLC = 0 << 1
FL_FLUX_FORCE = 1 << 1
FL_FLUX_LF = 2 << 1
FL_FLUX_RICHTMYER = 3 << 1
FL_LIMITER_VANLEER = 0 << 3
FL_LIMITER_SUPERBEE = 1 << 3
FL_RECON_MUSCL = 0 << 4
FL_RECON_BASIC = 1 << 4
FL_NO_FLATTEN = 1 << 5

FLUX_BITS = {"hllc": FL_FLUX_HLLC, "force": FL_FLUX_FORCE, "lf": FL_FLUX_LF,
             "richtmyer": FL_FLUX_RICHTMYER}
LIMITER_BITS = {"vanleer": FL_LIMITER_VANLEER, "superbee": FL_LIMITER_SUPERBEE}
RECON_BITS = {"muscl": FL_RECON_MUSCL, "basic": FL_RECON_BASIC}


class FlError(RuntimeError):
    """A C-ABI call returned a non-zero status."""

    def __init__(self, code: int, message: str):
        super().__init__(f"[fl status {code}] {message}")
        self.code = code


class Grid(C.Structure):
    _fields_ = [("dims", C.c_int32), ("n", C.c_int64 * 3), ("pitch", C.c_int64)]

    @staticmethod
    def make(shape, pitch: int | None = None) -> "Grid":
        """shape = (nx,), (nx, ny) or (nx, ny, nz), x first."""
        g = Grid()
        g.dims = len(shape)
        n = list(shape) + [1] * (3 - len(shape))
        for d in range(3):
            g.n[d] = int(n[d])
        cells = 1
        for v in shape:
            cells *= int(v)
        g.pitch = int(pitch if pitch is not None else cells)
        return g


def policy_bits(dtype: str = "f64", flux: str = "hllc", limiter: str = "vanleer",
                recon: str = "muscl", flatten: bool = True) -> int:
    bits = FL_DTYPE_F32 if dtype in ("f32", "float32", "float") else FL_DTYPE_F64
    bits |= FLUX_BITS[flux] | LIMITER_BITS[limiter] | RECON_BITS[recon]
    if not flatten:
        bits |= FL_NO_FLATTEN
    return bits


class Material(C.Structure):
    """fl_material: the ideal gas (p_inf = 0) or the stiffened fluid."""
    _fields_ = [("gamma", C.c_double), ("p_inf", C.c_double)]


class BatchDesc(C.Structure):
    _fields_ = [("dims", C.c_int32), ("n", C.c_int64 * 2), ("offset", C.c_int64),
                ("pitch", C.c_int64), ("res", C.c_double)]


# name -> (restype, argtypes); every symbol of include/fluidity_b200.h
_P = C.c_void_p
_G = C.POINTER(Grid)
PROTOTYPES = {
    "fl_version": (C.c_int, []),
    "fl_last_error_string": (C.c_char_p, []),
    "fl_policy_from_settings": (C.c_int, [C.c_char_p, C.POINTER(C.c_uint32),
                                          C.POINTER(C.c_int32)]),
    "fl_policy_from_settings_file": (C.c_int, [C.c_char_p, C.POINTER(C.c_uint32),
                                               C.POINTER(C.c_int32)]),
    "fl_state_bytes": (C.c_int64, [_G, C.c_uint32]),
    "fl_split_sweep_mat": (C.c_int, [_G, C.c_int, _P, _P, C.POINTER(Material), C.c_double,
                                     C.c_uint32, C.c_uint32, _P, _P]),
    "fl_split_solve_mat": (C.c_int, [_G, C.POINTER(_P), C.POINTER(_P), C.POINTER(Material),
                                     C.c_double, C.c_uint32, C.c_uint32, _P, _P]),
    "fl_max_wavespeed_mat": (C.c_int, [_G, _P, C.POINTER(Material), C.c_uint32, _P, _P]),
    "fl_workspace_bytes": (C.c_int64, [_G, C.c_uint32]),
    "fl_split_sweep_ws": (C.c_int, [_G, C.c_int, _P, _P, C.POINTER(Material), C.c_double,
                                    C.c_uint32, C.c_uint32, _P, _P, _P]),
    "fl_split_solve_ws": (C.c_int, [_G, C.POINTER(_P), C.POINTER(_P), C.POINTER(Material),
                                    C.c_double, C.c_uint32, C.c_uint32, _P, _P, _P]),
    "fl_workspace_status": (C.c_int, [_P, _P, C.POINTER(C.c_int)]),
    "fl_fill_riemann_mat": (C.c_int, [_G, _P, C.POINTER(Material), C.c_uint32, _P, _P]),
    "fl_sim_set_material": (C.c_int, [_P, C.POINTER(Material)]),
    "fl_host_pipe_create": (C.c_int, [C.POINTER(_P), _G, C.c_double, C.c_uint32, C.c_uint32,
                                      C.c_int]),
    "fl_host_pipe_destroy": (C.c_int, [_P]),
    "fl_host_pipe_set_material": (C.c_int, [_P, C.POINTER(Material)]),
    "fl_host_pipe_run": (C.c_int, [_P, C.c_int32, C.POINTER(_P), C.POINTER(_P), C.c_double,
                                   C.c_double, C.c_double, C.c_int64, C.POINTER(C.c_int64),
                                   C.POINTER(C.c_double)]),
    "fl_mm_set_materials": (C.c_int, [_P, C.POINTER(Material)]),
    "fl_mm_set_states_mat": (C.c_int, [_G, C.c_uint32, _P, _P, C.POINTER(C.c_double),
                                       C.POINTER(Material), _P]),
    "fl_split_sweep": (C.c_int, [_G, C.c_int, _P, _P, C.c_double, C.c_double, C.c_uint32,
                                 C.c_uint32, _P, _P]),
    "fl_split_solve": (C.c_int, [_G, C.POINTER(_P), C.POINTER(_P), C.c_double, C.c_double,
                                 C.c_uint32, C.c_uint32, _P, _P]),
    "fl_max_wavespeed": (C.c_int, [_G, _P, C.c_double, C.c_uint32, _P, _P]),
    "fl_fill_riemann": (C.c_int, [_G, _P, C.c_double, C.c_uint32, _P, _P]),
    "fl_aos_to_soa": (C.c_int, [_G, C.c_uint32, _P, _P, _P]),
    "fl_soa_to_aos": (C.c_int, [_G, C.c_uint32, _P, _P, _P]),
    "fl_sim_create": (C.c_int, [C.POINTER(_P), _G, C.c_double, C.c_uint32, C.c_uint32]),
    "fl_sim_destroy": (C.c_int, [_P]),
    "fl_sim_begin": (C.c_int, [_P, _P, _P, C.c_double, C.c_double, C.c_double, C.c_int64, _P]),
    "fl_sim_steps": (C.c_int, [_P, C.c_int64, _P]),
    "fl_sim_set_rows": (C.c_int, [_P, C.c_int64, C.c_int64]),
    "fl_sim_set_external_reduce": (C.c_int, [_P, C.c_int]),
    "fl_sim_set_ws_word": (C.c_int, [_P, _P]),
    "fl_sim_sweep": (C.c_int, [_P, C.c_int, _P]),
    "fl_sim_finalize": (C.c_int, [_P, C.c_int, _P]),
    "fl_sim_status": (C.c_int, [_P, _P, C.POINTER(C.c_int64), C.POINTER(C.c_double),
                                C.POINTER(C.c_int), C.POINTER(_P)]),
    "fl_slab_nccl_available": (C.c_int, []),
    "fl_slab_nccl_id": (C.c_int, [_P]),
    "fl_slab_create_nccl": (C.c_int, [C.POINTER(_P), _G, C.c_double, C.c_uint32, C.c_uint32,
                                      C.c_int64, C.c_int64, _P, C.c_int, C.c_int]),
    "fl_slab_create_local": (C.c_int, [C.POINTER(_P), _G, C.c_double, C.c_uint32, C.c_uint32,
                                       C.c_int64, C.c_int64]),
    "fl_slab_set_material": (C.c_int, [_P, C.POINTER(Material)]),
    "fl_slab_sim": (C.c_int, [_P, C.POINTER(_P)]),
    "fl_slab_begin": (C.c_int, [C.POINTER(_P), C.c_int, C.POINTER(_P), C.POINTER(_P), C.c_double,
                                C.c_double, C.c_double, C.c_int64, _P]),
    "fl_slab_steps": (C.c_int, [C.POINTER(_P), C.c_int, C.c_int64, _P]),
    "fl_slab_destroy": (C.c_int, [_P]),
    "fl_simulate": (C.c_int, [_P, _P, _P, C.c_double, C.c_double, C.c_double, C.c_int64, _P,
                              C.POINTER(C.c_int64), C.POINTER(C.c_double), C.POINTER(_P)]),
    "fl_simulate_noalloc": (C.c_int, [_G, C.c_double, C.c_uint32, C.c_uint32, _P, _P, C.c_double,
                                      C.c_double, C.c_double, C.c_int64, _P,
                                      C.POINTER(C.c_int64), C.POINTER(C.c_double),
                                      C.POINTER(_P)]),
    "fl_batch_create": (C.c_int, [C.POINTER(_P), C.POINTER(BatchDesc), C.c_int32, C.c_double,
                                  C.c_uint32, C.c_uint32]),
    "fl_batch_destroy": (C.c_int, [_P]),
    "fl_batch_set_material": (C.c_int, [_P, C.POINTER(Material)]),
    "fl_batch_begin": (C.c_int, [_P, _P, _P, C.c_double, C.c_double, C.c_int64, _P]),
    "fl_batch_steps": (C.c_int, [_P, C.c_int64, _P]),
    "fl_batch_capture": (C.c_int, [_P, C.c_int64]),
    "fl_batch_launch": (C.c_int, [_P, _P]),
    "fl_batch_status": (C.c_int, [_P, _P, C.POINTER(C.c_int64), C.POINTER(C.c_double),
                                  C.POINTER(C.c_int32)]),
    "fl_batch_autotune": (C.c_int, [_P, _P, _P, C.c_int64, _P]),
    "fl_batch_tuning": (C.c_int, [_P, C.POINTER(C.c_int32), C.c_int32]),
    "fl_adjoint_sweep": (C.c_int, [_G, C.c_int, _P, _P, _P, C.c_double, C.c_double, C.c_uint32,
                                   C.c_uint32, _P]),
    "fl_adj_create": (C.c_int, [C.POINTER(_P), _G, C.c_double, C.c_uint32, C.c_uint32,
                                C.c_int64, C.c_int64]),
    "fl_adjoint_sweep_mat": (C.c_int, [_G, C.c_int, _P, _P, _P, C.POINTER(Material), C.c_double,
                                       C.c_uint32, C.c_uint32, _P]),
    "fl_adj_destroy": (C.c_int, [_P]),
    "fl_adj_set_material": (C.c_int, [_P, C.POINTER(Material)]),
    "fl_adj_forward": (C.c_int, [_P, _P, _P, C.c_double, C.c_double, C.POINTER(C.c_double), _P]),
    "fl_adj_dtdh": (C.c_int, [_P, C.POINTER(C.c_double)]),
    "fl_adj_backward": (C.c_int, [_P, _P, _P, _P]),
    "fl_ls_workspace_bytes": (C.c_int64, [_G]),
    "fl_ls_velocity": (C.c_int, [_G, C.c_int, C.POINTER(_P), C.POINTER(_P), C.c_int64,
                                 C.c_uint32, C.c_double, _P, _P]),
    "fl_ls_advect": (C.c_int, [_G, _P, _P, C.c_double, C.c_double, _P, _P, _P]),
    "fl_ls_project": (C.c_int, [C.c_int64, _P, _P, _P]),
    "fl_ls_reinit": (C.c_int, [_G, _P, C.c_double, _P, _P, C.c_int, C.POINTER(C.c_int), _P]),
    "fl_mm_create": (C.c_int, [C.POINTER(_P), _G, C.POINTER(C.c_double), C.c_uint32,
                               C.c_double]),
    "fl_mm_destroy": (C.c_int, [_P]),
    "fl_mm_ghost": (C.c_int, [_P, _P, _P, _P, _P, _P, _P, C.c_int, _P]),
    "fl_mm_stats": (C.c_int, [_P, C.POINTER(C.c_int32), C.c_int32]),
    "fl_mm_set_states": (C.c_int, [_G, C.c_uint32, _P, _P, C.POINTER(C.c_double), C.c_double,
                                   _P]),
    "fl_mm_combine": (C.c_int, [_G, C.c_uint32, _P, _P, _P, _P]),
    "fl_mm_begin": (C.c_int, [_P, _P, _P, _P, _P, _P, _P, _P, _P, C.c_double, C.c_double,
                              C.c_int64, C.c_int]),
    "fl_mm_steps": (C.c_int, [_P, C.c_int64, _P]),
    "fl_mm_status": (C.c_int, [_P, _P, C.POINTER(C.c_int64), C.POINTER(C.c_double),
                               C.POINTER(C.c_int), C.POINTER(_P), C.POINTER(_P)]),
}

_lib = None


def load(path: str | None = None):
    """Load the library (built by fluidity_b200.build); raise if absent.
    FLUIDITY_B200_LIB names an alternative build of the same library."""
    global _lib
    if path is None:
        path = os.environ.get("FLUIDITY_B200_LIB", LIB_PATH)
    if _lib is not None and path == os.environ.get("FLUIDITY_B200_LIB", LIB_PATH):
        return _lib
    if not os.path.exists(path):
        raise ImportError(
            f"{path} is missing: build it with `python -m fluidity_b200.build` "
            "(the split solver has no CPU fallback)")
    lib = C.CDLL(path)
    for name, (res, args) in PROTOTYPES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path == os.environ.get("FLUIDITY_B200_LIB", LIB_PATH):
        _lib = lib
    return lib


def check(rc: int, lib=None) -> None:
    if rc != FL_OK:
        lib = lib or load()
        msg = lib.fl_last_error_string().decode(errors="replace")
        raise FlError(rc, msg)


def policy_from_settings(text: str):
    """(policy bits, dims) from a fluidity settings text's simulator block."""
    lib = load()
    pol = C.c_uint32()
    dims = C.c_int32()
    check(lib.fl_policy_from_settings(text.encode(), C.byref(pol), C.byref(dims)), lib)
    return int(pol.value), int(dims.value)
