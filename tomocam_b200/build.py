"""Build the native parts of tomocam_b200 in place.

* ``libtomocam_b200.so`` -- the CUDA kernels and the C ABI declared in
  ``include/tomocam_b200.h`` (nvcc, sm_100a only).
* ``cTomocam*.so`` -- the pybind11 module mirroring the reference's
  ``cTomocam`` (g++), linked against the C ABI library.

Usage: ``python -m tomocam_b200.build [--force] [--jobs N]``.
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
import sysconfig
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libtomocam_b200.so")

CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O2",
              "--expt-relaxed-constexpr", "-I" + INCLUDE, "-I" + CSRC]

CU_SOURCES = ["tc_fft.cu", "tc_nufft.cu", "tc_toeplitz.cu", "tc_toeplitz_fast.cu",
              "tc_prior.cu", "tc_prior_diff.cu", "tc_mbir.cu", "tc_batch.cu",
              "tc_prep.cu", "tc_capi.cu", "tc_noalloc.cu", "tc_hostio.cu", "tc_slab.cu",
              "tc_nufft_fast.cu"]


def _newer(target: str, deps) -> bool:
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(d) <= t for d in deps)


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    hs.append(os.path.join(INCLUDE, "tomocam_b200.h"))
    return hs


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    return r.stdout + r.stderr


def build_lib(force=False, jobs=8, verbose=False, extra=()):
    os.makedirs(BUILD, exist_ok=True)
    hdrs = _headers()
    objs, todo = [], []
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src.replace(".cu", ".o"))
        objs.append(o)
        if force or not _newer(o, [s] + hdrs):
            todo.append((s, o))

    def comp(so):
        s, o = so
        out = _run([NVCC, *ARCH, *NVCC_FLAGS, *extra, "-c", s, "-o", o])
        if verbose and out.strip():
            print(out)

    with ThreadPoolExecutor(max_workers=max(1, jobs)) as ex:
        list(ex.map(comp, todo))
    if todo or force or not _newer(LIB, objs):
        _run([NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"])
    return LIB


def build_pymod(force=False):
    import pybind11
    ext = sysconfig.get_config_var("EXT_SUFFIX") or ".so"
    out = os.path.join(HERE, "cTomocam" + ext)
    src = os.path.join(CSRC, "py_ctomocam.cpp")
    if not force and _newer(out, [src, LIB, os.path.join(INCLUDE, "tomocam_b200.h")]):
        return out
    cmd = ["g++", "-O2", "-shared", "-fPIC", "-std=c++17",
           "-I" + pybind11.get_include(), "-I" + sysconfig.get_paths()["include"],
           "-I" + INCLUDE, "-I" + os.path.join(CUDA_HOME, "include"), src, "-o", out,
           "-L" + HERE, "-ltomocam_b200", "-L" + os.path.join(CUDA_HOME, "lib64"), "-lcudart",
           "-Wl,-rpath,$ORIGIN", "-Wl,-rpath," + os.path.join(CUDA_HOME, "lib64")]
    _run(cmd)
    return out


def build(force=False, jobs=8, verbose=False):
    if not os.path.exists(NVCC):
        raise RuntimeError(f"nvcc not found at {NVCC}")
    lib = build_lib(force, jobs, verbose)
    mod = build_pymod(force)
    return lib, mod


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--jobs", type=int, default=8)
    ap.add_argument("--verbose", action="store_true")
    a = ap.parse_args(argv)
    for p in build(a.force, a.jobs, a.verbose):
        print(p)


if __name__ == "__main__":
    main()
