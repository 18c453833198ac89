"""Build the B200 extension in-tree.

* ``andosim_b200/lib/libando_gpu.so`` -- the CUDA kernels and the C ABI of
  ``include/ando_gpu.h`` (nvcc, sm_100a, static CUDA runtime).
* ``andosim_b200/ando_barrier_core*.so`` -- the pybind11 module with the
  reference's Python surface, linked against ``libando_gpu.so``.
"""
from __future__ import annotations

import os
import subprocess
import sys
import sysconfig
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIB = PKG / "lib"
CU_SOURCES = ["kernels.cu", "corrected.cu", "pcg.cu", "lbvh.cu", "learned.cu", "tc_gemm.cu", "capi.cu", "noalloc.cu", "diag.cu"]
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
              "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden", "--expt-relaxed-constexpr"]


def gpu_lib() -> Path:
    return LIB / "libando_gpu.so"


def py_ext() -> Path:
    return PKG / f"ando_barrier_core{sysconfig.get_config_var('EXT_SUFFIX') or '.so'}"


def _newer(out: Path, deps) -> bool:
    return out.exists() and all(out.stat().st_mtime >= Path(d).stat().st_mtime for d in deps)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(str(c) for c in cmd), file=sys.stderr)
    subprocess.run([str(c) for c in cmd], check=True)


def build(force: bool = False, verbose: bool = False) -> None:
    nvcc = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
    LIB.mkdir(exist_ok=True)
    headers = list(CSRC.glob("*.cuh")) + [ROOT / "include" / "ando_gpu.h"]
    objs = []
    jobs = []
    for src in CU_SOURCES:
        s = CSRC / src
        o = LIB / (s.stem + ".o")
        objs.append(o)
        if force or not _newer(o, [s] + headers):
            jobs.append([nvcc, *NVCC_FLAGS, "-c", s, "-o", o])
    with ThreadPoolExecutor(max_workers=len(jobs) or 1) as ex:
        list(ex.map(lambda c: _run(c, verbose), jobs))
    lib = gpu_lib()
    if force or jobs or not _newer(lib, objs):
        _run([nvcc, *NVCC_FLAGS, "-shared", *objs, "-o", lib, "-cudart", "static"], verbose)
    ext = py_ext()
    bsrc = CSRC / "bindings.cpp"
    if force or not _newer(ext, [bsrc, lib, ROOT / "include" / "ando_gpu.h"]):
        import pybind11
        cxx = os.environ.get("CXX", "g++")
        _run([cxx, "-O2", "-std=c++17", "-shared", "-fPIC", "-fvisibility=hidden",
              f"-I{pybind11.get_include()}", f"-I{sysconfig.get_paths()['include']}",
              bsrc, "-o", ext, f"-L{LIB}", "-lando_gpu", "-Wl,-rpath,$ORIGIN/lib"], verbose)


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(gpu_lib(), py_ext())
