"""Builds the mapp_b200 shared library for sm_100a with nvcc.

Usage: python -m mapp_b200.build  (or mapp_b200.build.build()).
The library is written in-tree as mapp_b200/libmapp_b200.so so it travels with
the source tree; object files go to mapp_b200/_build/.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libmapp_b200.so")
BUILD = os.path.join(HERE, "_build")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

SOURCES = ["mg_api.cu", "mg_atoms.cu", "mg_eam.cu", "mg_dmd.cu", "mg_dmd32.cu", "mg_mlp.cu", "mg_mlp_tc.cu", "mg_noalloc.cu", "mg_batch.cu", "mg_cfg.cu", "mg_md.cu", "mg_clock.cu"]
HEADERS = ["mg_internal.h", "mg_reduce.cuh", "mg_dmd_common.cuh", "mg_mlp_common.cuh", "mg_split.cuh"]

# a C++ client of the C ABI (the end-to-end measurement of bench.py)
CLIENT_SRC = os.path.join(HERE, "client", "mapp_e2e.cpp")
CLIENT = os.path.join(HERE, "mapp_e2e")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC,-ffp-contract=off",
         "-I" + os.path.join(HERE, "..", "include")]


def _stale(obj, deps):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, extra_flags=(), jobs: int = 4) -> str:
    os.makedirs(BUILD, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(HERE, "..", "include", "mapp_b200.h")]
    objs, procs = [], []
    for src in SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src.replace(".cu", ".o"))
        objs.append(o)
        if _stale(o, [s] + hdrs):
            cmd = [NVCC, *ARCH, *FLAGS, *extra_flags, "-c", s, "-o", o]
            if verbose:
                print(" ".join(cmd), flush=True)
            procs.append((subprocess.Popen(cmd), src))
            if len(procs) >= jobs:
                p, name = procs.pop(0)
                if p.wait() != 0:
                    raise RuntimeError(f"nvcc failed on {name}")
    for p, name in procs:
        if p.wait() != 0:
            raise RuntimeError(f"nvcc failed on {name}")
    if _stale(OUT, objs):
        cmd = [NVCC, *ARCH, "-shared", "-o", OUT, *objs, "-lcudart"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd)
    if _stale(CLIENT, [CLIENT_SRC, OUT, hdrs[-1]]):
        cmd = [NVCC, *ARCH, "-O2", "-std=c++17", "-cudart", "shared", "-I" + os.path.join(HERE, "..", "include"),
               CLIENT_SRC, "-o", CLIENT, "-L" + HERE, "-lmapp_b200", "-Xlinker", "-rpath,$ORIGIN"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd)
    return OUT


if __name__ == "__main__":
    build(verbose="-v" in sys.argv)
    print(OUT)
