#!/usr/bin/env python3
"""Builds liblxmfv.so (the C-ABI library with the sm_100a kernels) and the
lxmf-vanity command line tool, in-tree under lxmf-vanity_b200/.

    python lxmf-vanity_b200/build.py [--ptxas-verbose]

nvcc cross-compiles for sm_100a without a GPU; the CUDA runtime is linked
statically and OpenSSL's libcrypto dynamically (the recheck of every hit).
"""
from __future__ import annotations

import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
OBJ = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "liblxmfv.so")
CLI = os.path.join(PKG, "lxmf-vanity")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3"]
CXXFLAGS = ["-O3", "-fPIC", "-std=c++17", "-Wall", "-Wextra"]

CU_SOURCES = ["lxmfv.cu", "noalloc.cu", "pool.cu"]
CXX_SOURCES = ["host.cpp", "cpu_search.cpp"]
HEADERS = ["fe25519.cuh", "fe25519_ptx.cuh", "sha256_lxmf.cuh", "walk_kernels.cuh", "group_kernels.cuh", "ws_kernels.cuh",
           "prim_kernels.cuh",
           "cpu_sha256.h"]


def _run(cmd: list[str], verbose: bool) -> str:
    if verbose:
        print(" ".join(cmd), flush=True)
    p = subprocess.run(cmd, capture_output=True, text=True)
    if p.returncode != 0:
        sys.stderr.write(p.stdout + p.stderr)
        raise RuntimeError(f"build step failed: {' '.join(cmd[:3])} ...")
    return p.stdout + p.stderr


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, ptxas_verbose: bool = False, force: bool = False) -> str:
    """Compile what is out of date; returns the ptxas report when asked."""
    os.makedirs(OBJ, exist_ok=True)
    header_paths = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(ROOT, "include", "lxmfv.h")]
    objs = []
    report = ""
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ, src + ".o")
        objs.append(o)
        if force or ptxas_verbose or _stale(o, [s] + header_paths):
            extra = ["-Xptxas", "-v"] if ptxas_verbose else []
            report += _run([NVCC] + NVFLAGS + extra + ["-c", s, "-o", o], verbose)
    for src in CXX_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ, src + ".o")
        objs.append(o)
        if force or _stale(o, [s] + header_paths):
            _run(["g++"] + CXXFLAGS + ["-c", s, "-o", o], verbose)
    if force or _stale(LIB, objs):
        _run([NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcrypto"], verbose)
    cli_src = os.path.join(CSRC, "cli.cpp")
    if os.path.exists(cli_src) and (force or _stale(CLI, [cli_src, LIB] + header_paths)):
        _run(["g++"] + CXXFLAGS + [cli_src, "-o", CLI, "-L" + PKG, "-llxmfv", "-Wl,-rpath,$ORIGIN", "-lpthread"], verbose)
    return report


if __name__ == "__main__":
    rep = build(verbose=True, ptxas_verbose="--ptxas-verbose" in sys.argv, force="--force" in sys.argv)
    if rep:
        print(rep)
