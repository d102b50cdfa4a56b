"""Builds libdrpt_gpu.so in-tree with nvcc for sm_100a (B200) and the `drpt`
command-line host program.

    python -m drpt_b200.build            # library + CLI
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(PKG, "libdrpt_gpu.so")
CLI = os.path.join(PKG, "drpt")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                  "-Xcompiler", "-O2", "-Xptxas", "-O3", "--expt-relaxed-constexpr",
                  "-I" + INCLUDE, "-I" + CSRC]
# The reference-exact kernels reproduce the reference's FP32 operation
# sequences (projection sums, node statistics, medians, per-pair distances),
# so nothing in them may be contracted into a fused multiply-add; the other
# kernels (mixed form, FP32 Gram form, queries, learned splits) may.
EXACT_SOURCES = {"api.cu", "k_project.cu", "k_tree.cu", "k_local.cu", "k_leafknn.cu",
                 "k_merge.cu", "noalloc.cu", "host_algo.cpp"}


def _fmad_flag(src: str) -> str:
    return "-fmad=false" if os.path.basename(src) in EXACT_SOURCES else "-fmad=true"


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _host_cxx() -> str:
    # The system g++ (the one nvcc picks by default) is also the host compiler here.
    return "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"


def lib_sources() -> list[str]:
    return sorted(glob.glob(os.path.join(CSRC, "*.cu"))) + [os.path.join(CSRC, "host_algo.cpp")]


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build_library(force: bool = False, verbose: bool = False) -> str:
    deps = lib_sources() + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        glob.glob(os.path.join(CSRC, "*.h")) + [os.path.join(INCLUDE, "drpt_gpu.h")]
    if not force and not _stale(LIB, deps):
        return LIB
    objdir = os.path.join(PKG, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    for src in lib_sources():
        obj = os.path.join(objdir, os.path.basename(src) + ".o")
        cmd = [_nvcc(), "-ccbin", _host_cxx()] + NVFLAGS + [_fmad_flag(src), "-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
        objs.append(obj)
    cmd = [_nvcc(), "-ccbin", _host_cxx()] + ARCH + ["-shared", "-o", LIB] + objs
    subprocess.run(cmd, check=True)
    return LIB


def build_cli(force: bool = False) -> str:
    src = os.path.join(CSRC, "cli", "drpt_main.cpp")
    if not os.path.exists(src):
        return ""
    deps = [src, os.path.join(INCLUDE, "drpt_gpu.h"), LIB] + glob.glob(os.path.join(CSRC, "cli", "*"))
    if not force and not _stale(CLI, deps):
        return CLI
    cmd = [_host_cxx(), "-std=c++17", "-O2", "-I" + INCLUDE, "-I/usr/local/cuda/include", src,
           "-o", CLI, "-L" + PKG, "-ldrpt_gpu", "-Wl,-rpath,$ORIGIN", "-Wl,-Bstatic", "-lz",
           "-Wl,-Bdynamic"]
    subprocess.run(cmd, check=True)
    return CLI


def build_all(force: bool = False, verbose: bool = False) -> None:
    build_library(force=force, verbose=verbose)
    build_cli(force=force)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv, verbose="-v" in sys.argv)
