"""Builds libgbx.so (the sm_100a groupby kernels + C ABI) in-tree with nvcc.

Usage: python -m cudf_b200.build   (or cudf_b200.build.build_library()).
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libgbx.so")

SOURCES = ["gbx_kernels.cu", "gbx_warp.cu", "gbx_part.cu", "gbx_radix.cu", "gbx_tiled.cu", "gbx_batch.cu",
           "gbx_scan.cu", "gbx_stream.cu", "gbx_sort.cu", "gbx_distinct.cu", "gbx_rep.cu", "gbx_join.cu", "gbx_args.cu", "gbx_abi.cpp", "gbx_batch.cpp", "gbx_server.cpp", "gbx_noalloc.cu"]
HEADERS = ["gbx_plan.hpp", "gbx_host.hpp", "gbx_device.cuh", "gbx_table.cuh", "gbx_warpcore.cuh", "gbx_kernels.hpp",
           "gbx_batch.hpp", "gbx_scan.hpp", "gbx_sort.hpp", "gbx_rep.cuh", os.path.join("..", "..", "include", "gbx.h")]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
    "--expt-relaxed-constexpr",
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    for f in SOURCES + HEADERS:
        if os.path.getmtime(os.path.join(CSRC, f)) > t:
            return True
    return False


def build_library(force: bool = False, verbose: bool = False) -> str:
    if not force and not _stale():
        return LIB
    from concurrent.futures import ThreadPoolExecutor

    cmds, objs = [], []
    for src in SOURCES:
        obj = os.path.join(CSRC, "_build", src + ".o")
        os.makedirs(os.path.dirname(obj), exist_ok=True)
        lang = ["-x", "cu"] if src.endswith(".cpp") else []
        cmds.append([nvcc(), *lang, *NVCC_FLAGS, "-c", os.path.join(CSRC, src), "-o", obj])
        objs.append(obj)

    def compile_one(cmd):
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)

    with ThreadPoolExecutor(max_workers=max(1, min(len(cmds), os.cpu_count() or 1))) as ex:
        list(ex.map(compile_one, cmds))
    tmp = LIB + ".tmp"
    cmd = [nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", tmp, *objs]
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build_library(force="--force" in sys.argv, verbose=True))


FACADE_TEST_SRC = os.path.join(os.path.dirname(HERE), "tests", "cpp", "groupby_facade_test.cpp")
FACADE_TEST_BIN = os.path.join(os.path.dirname(HERE), "tests", "cpp", "_build", "groupby_facade_test")


def build_facade_test(verbose: bool = False) -> str:
    """Compiles the C++ facade test (reference-style gtests against include/cudf)."""
    os.makedirs(os.path.dirname(FACADE_TEST_BIN), exist_ok=True)
    inc = os.path.join(os.path.dirname(HERE), "include")
    cmd = [nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-std=c++17", "-O2", "-x", "cu", "-I", inc, FACADE_TEST_SRC, "-L", HERE, "-lgbx",
           "-Xlinker", "-rpath," + HERE, "-Xlinker", "-rpath,$ORIGIN/../../../cudf_b200", "-o", FACADE_TEST_BIN]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    return FACADE_TEST_BIN
