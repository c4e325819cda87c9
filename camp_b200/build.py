"""Builds libcamp_b200.so in-tree (camp_b200/libcamp_b200.so) for sm_100a.

    python -m camp_b200.build            # incremental
    python -m camp_b200.build --force    # rebuild everything

Host C++ is compiled by nvcc's host compiler; the CUDA runtime is linked
statically so the library only needs the driver at run time.
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libcamp_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CXXFLAGS = ["-O3", "-std=c++17", "-Xcompiler", "-fPIC,-Wall", "-lineinfo"]

SOURCES = ["model.cpp", "blob.cpp", "json.cpp", "loader.cpp", "capi.cpp", "serve.cpp", "solve.cu",
           "lanes.cu"]
HEADERS = ["model.hpp", "engine.hpp", "blob.hpp", "json.hpp", "loader.hpp", "serve.hpp",
           "bdf_consts.hpp", "rates.cuh", "block.cuh",
           os.path.join("..", "..", "include", "camp_b200.h")]


def _newer(src: str, dst: str) -> bool:
    return not os.path.exists(dst) or os.path.getmtime(src) > os.path.getmtime(dst)


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, h) for h in HEADERS]
    newest_header = max(os.path.getmtime(h) for h in headers)
    objs = []
    for src in SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if force or _newer(s, o) or os.path.getmtime(o) < newest_header:
            cmd = [NVCC, *ARCH, *CXXFLAGS, "-c", s, "-o", o]
            if src.endswith(".cu"):
                cmd += ["-Xptxas", "-v"] if verbose else []
            else:
                cmd += ["-x", "cu"] if src in ("capi.cpp", "serve.cpp") else []
            if verbose:
                print(" ".join(cmd))
            subprocess.run(cmd, check=True)
    if force or any(_newer(o, LIB) for o in objs):
        cmd = [NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-cudart", "static"]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose))
    sys.exit(0)
