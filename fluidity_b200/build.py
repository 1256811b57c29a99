"""Builds libfluidity_b200.so (the C ABI of include/fluidity_b200.h) in-tree.

Every translation unit under csrc/ is compiled for sm_100a only, in parallel,
then linked into one shared library next to this file.  Host code is compiled
with -ffp-contract=off so that host-side conversions round every product, as
the reference's host code does.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libfluidity_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
              "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
              "-Xptxas", "-O3"]
# The level-set velocity, projection and reinitialisation kernels and the
# ghost-fluid kernels keep every product separately rounded (no FMA
# contraction), so that they round exactly like the C restatement of the
# reference's arithmetic; the split-solver kernels and the level-set RK3
# stages (fl_ls_rk3.cu) contract freely.
FILE_FLAGS = {"fl_levelset.cu": ["--fmad=false"], "fl_mm.cu": ["--fmad=false"]}


def nvcc() -> str:
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    path = os.path.join(cuda, "bin", "nvcc")
    return path if os.path.exists(path) else (shutil.which("nvcc") or "nvcc")


def sources() -> list[str]:
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))


def _stale(lib: str, deps: list[str]) -> bool:
    if not os.path.exists(lib):
        return True
    t = os.path.getmtime(lib)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False, extra_flags: list[str] | None = None,
          lib: str = LIB) -> str:
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps.append(os.path.join(os.path.dirname(HERE), "include", "fluidity_b200.h"))
    deps.append(os.path.abspath(__file__))
    if not force and not _stale(lib, deps):
        return lib
    os.makedirs(BUILD, exist_ok=True)
    flags = NVCC_FLAGS + (extra_flags or [])
    tag = os.path.splitext(os.path.basename(lib))[0]

    def compile_one(src: str) -> str:
        obj = os.path.join(BUILD, f"{tag}_" + os.path.basename(src) + ".o")
        cmd = [nvcc(), *ARCH, *flags, *FILE_FLAGS.get(os.path.basename(src), []), "-c", src,
               "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src}:\n{r.stderr}")
        return obj

    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        objs = list(ex.map(compile_one, sources()))
    tmp = lib + ".tmp"
    cmd = [nvcc(), *ARCH, "-shared", "-o", tmp, *objs, "-lcudart", "-ldl"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stderr}")
    os.replace(tmp, lib)
    return lib


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
