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


def build(force=False, verbose=False):
    if not force and up_to_date():
        return LIB
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    nvcc = os.environ.get("NVCC", "nvcc")
    cmd = [nvcc, *ARCH, *FLAGS, "-o", LIB, *sources()]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if verbose or r.returncode:
        sys.stderr.write(r.stdout + r.stderr)
    if r.returncode:
        raise RuntimeError(f"nvcc failed ({r.returncode})")
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
