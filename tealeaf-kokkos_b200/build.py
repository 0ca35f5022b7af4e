"""Build recipe for the native parts of the package.

Products (all in this directory, built in-tree so they travel with the source tree):

* ``libtea2d_b200.so`` / ``libtea3d_b200.so`` -- the CUDA library behind the
  reference's ext_* C ABI (csrc/, compiled for sm_100a with -fmad=false so that every
  multiply and add rounds separately, as the reference's C++ does).
* ``libtea_driver.so`` and the ``tea_leaf`` executable -- the C++ restatement of the
  reference's Fortran driver (driver/).

Usage: ``python tealeaf-kokkos_b200/build.py`` or ``build()`` from Python.
"""
from __future__ import annotations

import os
import pathlib
import shutil
import subprocess
import sys

HERE = pathlib.Path(__file__).resolve().parent
CSRC = HERE / "csrc"
DRIVER = HERE / "driver"
INCLUDE = HERE.parent / "include"

NVCC_ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [
    "-O3", "-std=c++17", "-lineinfo", "-fmad=false",
    "-Xcompiler", "-fPIC,-ffp-contract=off,-fvisibility=hidden",
    f"-I{INCLUDE}",
]
HOST_CXX = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
HOST_FLAGS = ["-std=c++17", "-O2", "-fPIC", "-ffp-contract=off", "-Wall", "-Wextra"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the TeaLeaf B200 library needs the CUDA toolkit to build")


def _stale(target: pathlib.Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(pathlib.Path(d).stat().st_mtime > t for d in deps)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(str(c) for c in cmd), flush=True)
    subprocess.run([str(c) for c in cmd], check=True)


def cuda_sources():
    return sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cuh")) + sorted(INCLUDE.glob("*.h"))


def build(verbose: bool = False, force: bool = False) -> None:
    nvcc = _nvcc()
    cu = [CSRC / "tea_ext.cu", CSRC / "tea_fused.cu", CSRC / "tea_noalloc.cu", CSRC / "tea_warmstart.cu"]
    deps = cuda_sources()
    for dim in (2, 3):
        out = HERE / f"libtea{dim}d_b200.so"
        if force or _stale(out, deps):
            _run([nvcc, *NVCC_ARCH, *NVCC_FLAGS, f"-DTEA_DIM={dim}", "-shared", "-o", out, *cu], verbose)
    drv_deps = list(DRIVER.glob("*")) + sorted(INCLUDE.glob("*.h"))
    lib = HERE / "libtea_driver.so"
    if force or _stale(lib, drv_deps):
        _run([HOST_CXX, *HOST_FLAGS, "-shared", "-o", lib, DRIVER / "tea_driver.cpp", "-ldl"], verbose)
    exe = HERE / "tea_leaf"
    if force or _stale(exe, drv_deps + [lib]):
        _run([HOST_CXX, *HOST_FLAGS, "-o", exe, DRIVER / "tea_main.cpp", f"-L{HERE}", "-ltea_driver",
              "-Wl,-rpath,$ORIGIN"], verbose)


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv)
