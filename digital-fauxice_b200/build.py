#!/usr/bin/env python3
"""Build libfauxice_b200.so in-tree for sm_100a.

Numerics flags: --fmad=false (no FMA contraction), IEEE division and square
root, no fast math; host code also compiled with -ffp-contract=off.  The
library lands next to the Python package (fauxice_b200/), so it travels
with the source tree.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "fauxice_b200", "libfauxice_b200.so")
BUILD = os.path.join(HERE, "_build")
SOURCES = ("fx_analysis.cu", "fx_writer.cu", "fx_walk.cu", "fx_prelude.cu", "fx_api.cu",
           "fx_static.cu", "fx_route.cu", "fx_census.cu")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "--fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false",
    "-Xcompiler", "-fPIC,-ffp-contract=off,-fno-fast-math,-fvisibility=hidden",
    "-Xptxas", "-v",
]


def nvcc() -> str:
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(path):
        raise RuntimeError("nvcc not found")
    return path


def host_compiler() -> list[str]:
    # The environment may export a CC without a matching C++ runtime; use the
    # system g++ for nvcc's host side.
    gxx = shutil.which("g++")
    return ["-ccbin", gxx] if gxx else []


def build(verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    objects = []
    newest = 0.0
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    headers.append(os.path.join(os.path.dirname(HERE), "include", "fauxice_b200.h"))
    header_time = max(os.path.getmtime(h) for h in headers)
    for src in SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(BUILD, src.replace(".cu", ".o"))
        objects.append(obj)
        stale = (not os.path.exists(obj) or os.path.getmtime(obj) < max(os.path.getmtime(path),
                                                                        header_time))
        if stale:
            cmd = [nvcc(), *host_compiler(), *NVCC_FLAGS, "-c", path, "-o", obj]
            res = subprocess.run(cmd, capture_output=True, text=True)
            log = res.stdout + res.stderr
            if verbose or res.returncode:
                sys.stderr.write(log)
            with open(obj + ".log", "w") as handle:
                handle.write(log)
            if res.returncode:
                raise RuntimeError(f"nvcc failed for {src}")
        newest = max(newest, os.path.getmtime(obj))
    if not os.path.exists(OUT) or os.path.getmtime(OUT) < newest:
        cmd = [nvcc(), *host_compiler(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared",
               "-o", OUT, *objects, "-lcudart", "-lcrypto"]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode:
            sys.stderr.write(res.stdout + res.stderr)
            raise RuntimeError("link failed")
    return OUT


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
