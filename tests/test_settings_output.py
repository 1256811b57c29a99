"""Settings-file dispatch (fl_policy_from_settings, the run-time form of the
reference's Settings::from_string + OptionManager::create) and the
one-file-per-variable raw output (SimulatorImpl::write_results_separate_raw).

Choice strings follow the reference's option headers
(setting/data_option.hpp:40, dimension_option.hpp:43, limiter_option.hpp:46,
reconstruction_option.hpp:44, flux_method_option.hpp:44,
material_option.hpp:43, limit_form_option.hpp:42, solve_option.hpp:44,
execution_option.hpp:41); the example text has the layout of the reference's
validation settings files."""
import ctypes as C
import os

import numpy as np
import pytest

from fluidity_b200 import capi
from fluidity_b200.solver import SimulatorImpl, write_separate_raw

EXAMPLE = """{
  simulator : {
    data_type     : double,
    material      : ideal-gas,
    limit_form    : conservative,
    limiter       : van-leer,
    reconstructor : muscl-hancock,
    flux_method   : force,
    solve_method  : split,
    execution     : gpu
  },
  cfl         : 0.9,
  shock       : {
    x    : 0.1,
    mach : 1.22
  },
  domain : {
   resolution : 0.001,
   x          : { start : 0.0, end : 1.6 },
   y          : { start : 0.0, end : 1.0 }
  }
}
"""


def sim_block(**entries):
    body = ",\n".join(f"  {k} : {v}" for k, v in entries.items())
    return "simulator : {\n" + body + "\n}\n"


def test_example_settings_file_text():
    pol, dims = capi.policy_from_settings(EXAMPLE)
    assert pol == capi.FL_DTYPE_F64 | capi.FL_LIMITER_VANLEER | capi.FL_RECON_MUSCL | \
        capi.FL_FLUX_FORCE
    assert dims == 1


def test_defaults_follow_sim_traits():
    # SimTraits (simulator/simulator_traits.hpp:44-58): double, 1-D, Superbee,
    # MUSCL-Hancock, FORCE
    pol, dims = capi.policy_from_settings("simulator : { }")
    assert pol == capi.FL_DTYPE_F64 | capi.FL_LIMITER_SUPERBEE | capi.FL_RECON_MUSCL | \
        capi.FL_FLUX_FORCE
    assert dims == 1


@pytest.mark.parametrize("key,value,mask,bits", [
    ("data_type", "float", 1, capi.FL_DTYPE_F32),
    ("data_type", "double", 1, capi.FL_DTYPE_F64),
    ("limiter", "van-leer", 1 << 3, capi.FL_LIMITER_VANLEER),
    ("limiter", "superbee", 1 << 3, capi.FL_LIMITER_SUPERBEE),
    ("reconstructor", "none", 1 << 4, capi.FL_RECON_BASIC),
    ("reconstructor", "muscl-hancock", 1 << 4, capi.FL_RECON_MUSCL),
    ("flux_method", "force", 3 << 1, capi.FL_FLUX_FORCE),
    ("flux_method", "hllc", 3 << 1, capi.FL_FLUX_HLLC),
    ("flux_method", "lax-friedrichs", 3 << 1, capi.FL_FLUX_LF),
    ("flux_method", "richtmyer", 3 << 1, capi.FL_FLUX_RICHTMYER),
])
def test_each_choice(key, value, mask, bits):
    pol, _ = capi.policy_from_settings(sim_block(**{key: value}))
    assert pol & mask == bits


@pytest.mark.parametrize("word,dims", [("one", 1), ("two", 2), ("three", 3)])
def test_dimensions(word, dims):
    assert capi.policy_from_settings(sim_block(dimensions=word))[1] == dims


def test_comments_and_whitespace():
    text = ("# a comment line with simulator : { data_type : float }\n"
            "simulator:{data_type:float,\n"
            "   # flux_method : hllc\n"
            "\tflux_method :   richtmyer  ,dimensions:three}\n")
    pol, dims = capi.policy_from_settings(text)
    assert pol & 1 == capi.FL_DTYPE_F32
    assert pol & (3 << 1) == capi.FL_FLUX_RICHTMYER
    assert dims == 3


@pytest.mark.parametrize("text,needle", [
    ("cfl : 0.9", "no 'simulator"),
    (sim_block(limiter="linear"), "unsupported limiter 'linear'"),
    (sim_block(limiter="void"), "unsupported limiter"),
    (sim_block(limit_form="primitive"), "unsupported limit_form"),
    (sim_block(solve_method="unsplit"), "unsupported solve_method"),
    (sim_block(material="stiff-fluid"), "unsupported material"),
    (sim_block(data_type="half"), "unsupported data_type"),
    (sim_block(dimensions="four"), "unsupported dimensions"),
    (sim_block(execution="cpu"), "unsupported execution"),
    (sim_block(flux_metod="hllc"), "unknown simulator setting 'flux_metod'"),
    ("simulator : double", "must be { name : value"),
])
def test_rejected_settings(text, needle):
    with pytest.raises(capi.FlError) as e:
        capi.policy_from_settings(text)
    assert e.value.code == capi.FL_EINVAL
    assert needle in str(e.value)


def test_settings_file(tmp_path):
    lib = capi.load()
    path = tmp_path / "settings.txt"
    path.write_text(EXAMPLE.replace("van-leer", "superbee").replace("force", "hllc"))
    pol, dims = C.c_uint32(), C.c_int32()
    capi.check(lib.fl_policy_from_settings_file(str(path).encode(), C.byref(pol),
                                                C.byref(dims)), lib)
    assert pol.value == capi.FL_DTYPE_F64 | capi.FL_LIMITER_SUPERBEE | capi.FL_RECON_MUSCL | \
        capi.FL_FLUX_HLLC
    rc = lib.fl_policy_from_settings_file(str(tmp_path / "missing.txt").encode(),
                                          C.byref(pol), C.byref(dims))
    assert rc != 0
    assert b"cannot open" in lib.fl_last_error_string()
    assert lib.fl_policy_from_settings(None, C.byref(pol), C.byref(dims)) != 0


def test_simulator_from_settings():
    sim = SimulatorImpl.from_settings(sim_block(data_type="float", dimensions="two",
                                                limiter="van-leer", flux_method="hllc",
                                                reconstructor="none"), gamma=1.4)
    assert sim.dims == 2
    assert sim.kw["dtype"] == "f32"
    assert sim.kw["flux"] == "hllc"
    assert sim.kw["limiter"] == "vanleer"
    assert sim.kw["recon"] == "basic"
    sim = SimulatorImpl.from_settings(EXAMPLE)
    assert (sim.dims, sim.kw["dtype"], sim.kw["flux"], sim.kw["limiter"], sim.kw["recon"]) == \
        (1, "f64", "force", "vanleer", "muscl")


def _state(shape, dtype, seed):
    rng = np.random.default_rng(seed)
    D = len(shape)
    cells = int(np.prod(shape))
    rho = rng.uniform(0.5, 2.0, cells)
    vel = rng.uniform(-1.0, 1.0, (D, cells))
    p = rng.uniform(0.2, 3.0, cells)
    u = np.zeros((D + 2, cells + 7))                   # padded like a pitched plane
    u[0, :cells] = rho
    u[1, :cells] = p / 0.4 + 0.5 * rho * np.sum(vel * vel, axis=0)
    u[2:, :cells] = rho * vel
    return u.astype(dtype), rho, p, vel


@pytest.mark.parametrize("shape", [(5,), (4, 3), (3, 2, 2)])
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_separate_raw_layout(tmp_path, shape, dtype):
    D = len(shape)
    u, rho, p, vel = _state(shape, dtype, 3 + D)
    prefix = str(tmp_path / "out")
    paths = write_separate_raw(u, shape, 1.4, prefix, 0.25)
    names = ["rho", "p", "v_x", "v_y", "v_z"][:D + 2]
    nz = shape[2] if D == 3 else 1
    if D == 3:
        expect = [f"{prefix}_{z}_{n}_0.250000.dat" for z in range(nz) for n in names]
    else:
        expect = [f"{prefix}_{n}_0.250000.dat" for n in names]
    assert paths == expect
    assert all(os.path.exists(q) for q in expect)
    truth = [rho, p] + list(vel)
    tol = 1e-5                                     # %g keeps 6 significant digits
    ny = shape[1] if D >= 2 else 1
    for z in range(nz):
        for k, n in enumerate(names):
            path = expect[z * len(names) + k]
            text = open(path).read()
            lines = text.split("\n")
            if D == 1:
                assert text.endswith("\n\n") and lines[1] == ""
            else:
                assert len(lines) == ny + 1 and lines[-1] == ""
            for y in range(ny):
                assert lines[y].endswith(" ")
                vals = np.array([float(t) for t in lines[y].split()])
                assert len(vals) == shape[0]
                ref = truth[k].reshape(nz, ny, shape[0])[z, y]
                assert np.allclose(vals, ref, rtol=tol, atol=1e-5)
                if dtype == np.float64 and k == 0:       # density is stored as is
                    assert lines[y].split() == ["%g" % r for r in ref]
