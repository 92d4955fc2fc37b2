"""Builds libdcrf_cuda.so (sm_100a) in-tree with nvcc.

``python -m densecrf_ho_b200.build`` or ``build()`` from Python.  Objects go
to ``densecrf_ho_b200/_build/``; the shared library to
``densecrf_ho_b200/libdcrf_cuda.so``.  Every translation unit is compiled with
``-fmad=false`` so that no multiply-add is contracted: the reference's SSE2
arithmetic rounds each product and sum separately, and the library
reproduces it bit for bit.
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libdcrf_cuda.so")
INCLUDE = os.path.join(ROOT, "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-fmad=false", "-Xcompiler", "-fPIC",
              "--expt-relaxed-constexpr", "-I", INCLUDE, "-I", CSRC]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def _deps():
    return _sources() + glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(INCLUDE, "*.h"))


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(p) <= t for p in _deps())


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and up_to_date():
        return LIB
    os.makedirs(BUILD, exist_ok=True)
    exe = nvcc()
    hdr_t = max(os.path.getmtime(p) for p in _deps())

    def compile_one(src):
        obj = os.path.join(BUILD, os.path.basename(src)[:-3] + ".o")
        if not force and os.path.exists(obj) and os.path.getmtime(obj) >= max(hdr_t, os.path.getmtime(src)):
            return obj
        cmd = [exe, *ARCH, *NVCC_FLAGS, "-c", src, "-o", obj]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
        if verbose and r.stderr:
            sys.stderr.write(r.stderr)
        return obj

    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(compile_one, _sources()))
    tmp = LIB + ".tmp"
    r = subprocess.run([exe, *ARCH, "-shared", "-o", tmp, *objs, "-lcudart"], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, LIB)
    return LIB


SHIM_DIR = os.path.join(PKG, "cpp")
SHIM_BIN = os.path.join(SHIM_DIR, "shim_selftest")
CLI_BIN = os.path.join(SHIM_DIR, "example_inference")


def _build_cpp(src_name: str, out: str, eigen_include: str) -> str:
    lib = build()
    src = os.path.join(SHIM_DIR, src_name)
    deps = [src] + glob.glob(os.path.join(SHIM_DIR, "*.h")) + [lib]
    if os.path.exists(out) and all(os.path.getmtime(p) <= os.path.getmtime(out) for p in deps):
        return out
    cmd = ["g++", "-std=c++14", "-O2", "-w", "-I", INCLUDE, "-I", SHIM_DIR, "-I", eigen_include,
           "-I", "/usr/local/cuda/include", src, "-o", out, "-L", PKG, "-ldcrf_cuda",
           "-Wl,-rpath,$ORIGIN/.."]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"{src_name} build failed:\n{r.stderr}")
    return out


def build_shim(eigen_include: str) -> str:
    """Compiles the drop-in C++ API self-test and the headless example program
    (densecrf_ho_b200/cpp) with g++ against `eigen_include` (a directory
    holding Eigen/Core, e.g. the one the reference vendors) and
    libdcrf_cuda.so."""
    _build_cpp("example_inference.cpp", CLI_BIN, eigen_include)
    return _build_cpp("shim_selftest.cpp", SHIM_BIN, eigen_include)


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
