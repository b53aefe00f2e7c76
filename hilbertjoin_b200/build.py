"""Builds the engine in-tree: ``lib/libhj.so`` (CUDA, sm_100a) and the two
command-line executables ``bin/hilbertSelfJoinCardinality`` and
``bin/hilbertJoinCardinality``. nvcc cross-compiles without a GPU.

    python -m hilbertjoin_b200.build
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "lib", "libhj.so")
BIN = os.path.join(HERE, "bin")

CU_SOURCES = ["hj_engine.cu", "hj_prep.cu", "hj_index.cu", "hj_join_fp64.cu", "hj_join_tc.cu", "hj_server.cu",
              "hj_noalloc.cu", "hj_batch.cu"]
GENCODE = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
              "--expt-relaxed-constexpr"]


def _nvcc() -> str:
    for p in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if p and (os.path.isabs(p) and os.path.exists(p) or not os.path.isabs(p)):
            return p
    return "nvcc"


def _newer(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build_lib(verbose: bool = False, force: bool = False) -> str:
    """Compiles every CUDA source to an object (in parallel; a source is
    recompiled when it, a header or the C ABI changed) and links libhj.so."""
    from concurrent.futures import ThreadPoolExecutor
    srcs = [os.path.join(CSRC, s) for s in CU_SOURCES if os.path.exists(os.path.join(CSRC, s))]
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(ROOT, "include", "hj.h"))
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = [os.path.join(objdir, os.path.basename(s)[:-3] + ".o") for s in srcs]
    todo = [(s, o) for s, o in zip(srcs, objs) if force or _newer(o, [s, *headers])]
    if not todo and not _newer(LIB, objs):
        return LIB
    os.makedirs(os.path.dirname(LIB), exist_ok=True)

    def compile_one(so):
        s, o = so
        cmd = [_nvcc(), *GENCODE, *NVCC_FLAGS, "-c", "-o", o + ".tmp", s]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
        os.replace(o + ".tmp", o)

    with ThreadPoolExecutor(max_workers=min(8, max(1, len(todo)))) as ex:
        list(ex.map(compile_one, todo))
    cmd = [_nvcc(), *GENCODE, "-shared", "-o", LIB + ".tmp", *objs, "-lpthread"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


def build_cli(verbose: bool = False, force: bool = False) -> list:
    src = os.path.join(HERE, "cli", "hj_cli.cpp")
    if not os.path.exists(src):
        return []
    os.makedirs(BIN, exist_ok=True)
    outs = []
    for name, mode in (("hilbertSelfJoinCardinality", "HJ_CLI_SELF"), ("hilbertJoinCardinality", "HJ_CLI_JOIN")):
        exe = os.path.join(BIN, name)
        outs.append(exe)
        if not force and not _newer(exe, [src, LIB, os.path.join(ROOT, "include", "hj.h")]):
            continue
        cmd = ["g++", "-O2", "-std=c++17", f"-D{mode}", "-I", os.path.join(ROOT, "include"), "-o", exe, src,
               "-L", os.path.dirname(LIB), "-lhj", f"-Wl,-rpath,$ORIGIN/../lib", "-lpthread"]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return outs


def build(verbose: bool = False, force: bool = False) -> None:
    build_lib(verbose, force)
    build_cli(verbose, force)


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv)
