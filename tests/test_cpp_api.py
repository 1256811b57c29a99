"""The C++ policy interface (include/fluidity_b200/fluidity.hpp): a program
written like the reference's validation mains compiles against it, and its
GPU result matches the oracle."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")


def compile_program(tmp_path, name="toro_case1"):
    from fluidity_b200 import build
    lib = build.build()
    exe = str(tmp_path / name)
    cmd = ["g++", "-O2", "-std=c++17", os.path.join(ROOT, "tests", "cpp", name + ".cpp"),
           f"-I{os.path.join(ROOT, 'include')}", f"-I{CUDA}/include",
           f"-L{os.path.dirname(lib)}", "-lfluidity_b200", f"-L{CUDA}/lib64", "-lcudart",
           f"-Wl,-rpath,{os.path.dirname(lib)}", "-o", exe]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe


@pytest.mark.parametrize("name", ["toro_case1", "stiff_tube"])
def test_cpp_interface_compiles(tmp_path, name):
    assert os.path.exists(compile_program(tmp_path, name))


@pytest.mark.gpu
def test_cpp_toro_case1_matches_oracle(cuda, oracle, tmp_path):
    exe = compile_program(tmp_path)
    out = subprocess.run([exe, str(tmp_path / "toro1")], check=True, capture_output=True,
                         text=True).stdout
    iters = int(out.split()[1])
    data = np.loadtxt(str(tmp_path / "toro1.dat"))
    n = 400
    pos = np.arange(n, dtype=np.float32) / np.float32(n)
    left = pos < 0.3
    prim = np.vstack([np.where(left, 1.0, 0.125), np.where(left, 1.0, 0.1),
                      np.where(left, 0.75, 0.0)])
    u = oracle.prim_to_cons(prim, 1.4)
    ref, steps, rt, _ = oracle.simulate((n,), u, 1.4, 0.9, 0.0025, 0.2, 10 ** 9)
    assert iters == steps
    rp = oracle.cons_to_prim(ref, 1.4)
    got = data[:, 1:].T                    # rho, p, v_x
    assert np.max(np.abs(got - rp) / np.maximum(np.abs(rp), 1e-3)) < 1e-9
    for k, name in enumerate(["rho", "p", "v_x"]):
        text = open(str(tmp_path / f"toro1_raw_{name}_0.200000.dat")).read()
        assert text.endswith(" \n\n")
        vals = np.array([float(t) for t in text.split()])
        assert vals.shape == (n,)
        assert np.allclose(vals, rp[k], rtol=1e-5, atol=1e-6)


@pytest.mark.gpu
def test_cpp_stiff_tube_matches_oracle(cuda, oracle, tmp_path):
    """material::StiffFluid<double>{4.4} (p_inf = 0.613, as the reference's
    one-argument constructor leaves it) through SimulatorImpl."""
    exe = compile_program(tmp_path, "stiff_tube")
    out = subprocess.run([exe, str(tmp_path / "stiff")], check=True, capture_output=True,
                         text=True).stdout
    iters = int(out.split()[1])
    data = np.loadtxt(str(tmp_path / "stiff.dat"))
    n = 200
    with oracle.stiffened(0.613):
        u = oracle.fill_riemann((n,), np.array([[1.0, 10.0, 0.0], [1.0, 1.0, 0.0]]), 4.4)
        ref, steps, rt, _ = oracle.simulate((n,), u, 4.4, 0.9, 0.005, 0.05, 10 ** 9)
    assert iters == steps
    rp = oracle.cons_to_prim(ref, 4.4)     # pressure read back as p + gamma p_inf
    got = data[:, 1:].T
    assert np.max(np.abs(got - rp) / np.maximum(np.abs(rp), 1e-3)) < 1e-9
