"""Build the in-tree CUDA library (libctl.so) and the `cutauleaping` CLI.

Both are compiled for sm_100a only and land next to this file, so that a
checkout carries its own native code (no JIT cache, no site-packages).

    python -m cutauleaping_b200.build
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
LIB = os.path.join(HERE, "libctl.so")
CLI = os.path.join(HERE, "cutauleaping")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# -fmad=false: no implicit FMA contraction, so FP32/FP64 results match the
# reference arithmetic contract bit for bit (explicit fma() stays fused).
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-fmad=false", "-std=c++17",
                     "-Xcompiler", "-fPIC,-ffp-contract=off,-O3", f"-I{INCLUDE}"]

LIB_SOURCES = ["ctl_sweep.cu", "ctl_mlp.cu", "ctl_host.cpp"]
CLI_SOURCES = ["ctl_cli.cpp"]


def _newer(target: str, sources) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    deps = list(sources) + [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + \
        [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE)]
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build(force: bool = False, verbose: bool = False) -> None:
    srcs = [os.path.join(CSRC, s) for s in LIB_SOURCES]
    if force or _newer(LIB, srcs):
        _run(["nvcc", *NVCC_FLAGS, "-shared", "-o", LIB, *srcs], verbose)
    cli_srcs = [os.path.join(CSRC, s) for s in CLI_SOURCES]
    if force or _newer(CLI, cli_srcs + [LIB]):
        _run(["g++", "-O2", "-std=c++17", f"-I{INCLUDE}", "-o", CLI, *cli_srcs,
              f"-L{HERE}", "-lctl", "-Wl,-rpath,$ORIGIN"], verbose)


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
