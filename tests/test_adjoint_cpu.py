"""CPU check of the hand-written reverse mode (fluidity_b200/csrc/fl_adjoint.cuh):
tests/cpp/adjoint_fd.cpp compares every reverse function (physical flux,
HLLC in all wave regions, FORCE, MUSCL-Hancock evolution) with central finite
differences on random states."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_adjoint_primitives_match_finite_differences(tmp_path):
    exe = str(tmp_path / "adjoint_fd")
    subprocess.run(["g++", "-O2", "-std=c++17", f"-I{ROOT}",
                    os.path.join(ROOT, "tests", "cpp", "adjoint_fd.cpp"), "-o", exe],
                   check=True, capture_output=True, text=True)
    r = subprocess.run([exe], capture_output=True, text=True)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
