"""Build the native library libb200ldl.so in-tree for sm_100a.

    python -m amigo_b200.build          # incremental
    python -m amigo_b200.build --force  # rebuild everything

The library lands next to this file (amigo_b200/libb200ldl.so) so that it
travels with the working tree; nothing is installed into site-packages.
"""

from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
ROOT = os.path.dirname(HERE)
BUILD = os.path.join(ROOT, "_build")
LIB = os.path.join(HERE, "libb200ldl.so")

SOURCES = ["symbolic.cpp", "api.cu", "factor.cu", "solve.cu", "big.cu", "cluster_front.cu", "big_chain.cu", "noalloc.cu", "refine.cu", "solve_big.cu", "batch.cu", "assembly.cu", "big_app.cu", "schur_tc.cu"]
HEADERS = ["symbolic.h", "ldl_internal.h", "front_common.cuh", "umma.cuh"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    cand = os.environ.get("NVCC") or shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    return cand


def _host_cxx() -> list[str]:
    # nvcc needs a g++ it accepts; prefer the system driver
    for c in ("/usr/bin/g++-13", "/usr/bin/g++"):
        if os.path.exists(c):
            return ["-ccbin", c]
    return []


def _stale(obj: str, src: str) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    deps = [src] + [os.path.join(CSRC, h) for h in HEADERS]
    deps.append(os.path.join(ROOT, "include", "b200ldl.h"))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    objs = []
    common = ["-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-lineinfo"] + ARCH + _host_cxx()
    for src in SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(BUILD, src + ".o")
        objs.append(obj)
        if force or _stale(obj, path):
            cmd = [nvcc(), "-c", path, "-o", obj] + common
            if src.endswith(".cpp"):
                cmd = [nvcc(), "-x", "c++", "-c", path, "-o", obj] + common
            if verbose:
                print(" ".join(cmd))
            subprocess.run(cmd, check=True)
    if force or not os.path.exists(LIB) or any(
        os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs
    ):
        cmd = [nvcc(), "-shared", "-o", LIB] + objs + ARCH + _host_cxx() + ["-lcudart"]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return LIB


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args(argv)
    print(build(force=a.force, verbose=a.verbose))
    return 0


if __name__ == "__main__":
    sys.exit(main())
