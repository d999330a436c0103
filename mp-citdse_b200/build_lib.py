"""Builds libmpc_tdse.so in-tree for sm_100a (nvcc, no JIT cache).

Usage: python mp-citdse_b200/build_lib.py  (or __graft_entry__.build()).
Rebuilds only when a source under csrc/ or include/ is newer than the
library.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
LIB = os.path.join(PKG, "lib", "libmpc_tdse.so")
HOSTLIB = os.path.join(PKG, "lib", "libmpc_host.so")
TDSE = os.path.join(PKG, "bin", "tdse")
# the system C++ compiler (an environment CXX may link libstdc++ statically,
# which breaks iostreams inside a library loaded by Python)
CXX = "g++"
# NVTX (header-only) for the executable's profiler ranges
CUDA_INCLUDE = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "include")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-shared",
         "-Xptxas", "-v", "--expt-relaxed-constexpr"]


def sources():
    return sorted(glob.glob(os.path.join(PKG, "csrc", "*.cu")))


def deps():
    return (sources() + glob.glob(os.path.join(PKG, "csrc", "*.cuh")) +
            glob.glob(os.path.join(PKG, "csrc", "*.h")) +
            glob.glob(os.path.join(ROOT, "include", "*.h")))


def up_to_date():
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(d) <= t for d in deps())


def host_sources():
    return sorted(glob.glob(os.path.join(PKG, "host", "*")))


def _newer(target, deps_):
    return os.path.exists(target) and all(os.path.getmtime(d) <= os.path.getmtime(target)
                                          for d in deps_)


def build_host(force=False, verbose=False):
    """libmpc_host.so (HDF5 subset) and the drop-in `tdse` executable."""
    os.makedirs(os.path.dirname(TDSE), exist_ok=True)
    hdeps = host_sources() + glob.glob(os.path.join(ROOT, "include", "*.h"))
    jobs = []
    if force or not _newer(HOSTLIB, hdeps):
        jobs.append([CXX, "-std=c++17", "-O2", "-fPIC", "-shared", "-o", HOSTLIB,
                     os.path.join(PKG, "host", "h5lite.cpp"),
                     os.path.join(PKG, "host", "host_abi.cpp")])
    if force or not _newer(TDSE, hdeps + [LIB]):
        jobs.append([CXX, "-std=c++17", "-O2", "-o", TDSE,
                     os.path.join(PKG, "host", "tdse_main.cpp"),
                     os.path.join(PKG, "host", "h5lite.cpp"),
                     "-I", os.path.join(ROOT, "include"), "-I", CUDA_INCLUDE,
                     "-L", os.path.dirname(LIB), "-lmpc_tdse",
                     "-Wl,-rpath,$ORIGIN/../lib"])
    for cmd in jobs:
        r = subprocess.run(cmd, capture_output=True, text=True)
        if verbose or r.returncode:
            sys.stderr.write(r.stdout + r.stderr)
        if r.returncode:
            raise RuntimeError(f"{cmd[0]} failed ({r.returncode})")


def build(force=False, verbose=False):
    if not force and up_to_date():
        build_host(force, verbose)
        return LIB
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    nvcc = os.environ.get("NVCC", "nvcc")
    cmd = [nvcc, *ARCH, *FLAGS, "-o", LIB, *sources()]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if verbose or r.returncode:
        sys.stderr.write(r.stdout + r.stderr)
    if r.returncode:
        raise RuntimeError(f"nvcc failed ({r.returncode})")
    build_host(force, verbose)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
