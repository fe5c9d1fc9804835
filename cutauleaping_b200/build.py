"""Build the in-tree CUDA library (libctl.so) and the `cutauleaping` CLI.

Both are compiled for sm_100a only and land next to this file, so that a
checkout carries its own native code (no JIT cache, no site-packages).

    python -m cutauleaping_b200.build
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

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

GROUP_SIZES = (1, 2, 4, 8, 16, 32, 64, 128, 256)
LIB_SOURCES = (["ctl_sweep.cu", "ctl_tiny.cu", "ctl_mlp.cu", "ctl_host.cpp"] +
               [f"ctl_sweep_g{g}.cu" for g in GROUP_SIZES])
OBJ = os.path.join(HERE, "_obj")
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


# Headers that the library also hands to NVRTC at run time, to compile
# kernels specialised for one network (ctl_tiny.cu, ctl_sweep.cu): embedded
# as strings.
EMBEDDED = (("ctl_src_devmath", "ctl_devmath.cuh"), ("ctl_src_tiny_body", "ctl_tiny_body.cuh"),
            ("ctl_src_sweep_dev", "ctl_sweep_dev.cuh"))


def _embed_sources(path: str) -> None:
    parts = ["// Generated by cutauleaping_b200/build.py: device sources for NVRTC.", "namespace ctl {"]
    for sym, name in EMBEDDED:
        text = open(os.path.join(CSRC, name)).read()
        if ")CTLSRC\"" in text:
            raise RuntimeError(f"{name} contains the raw-string delimiter")
        parts.append(f'extern const char* const {sym} = R"CTLSRC({text})CTLSRC";')
    parts.append("}  // namespace ctl")
    open(path, "w").write("\n".join(parts) + "\n")


def build(force: bool = False, verbose: bool = False) -> None:
    srcs = [os.path.join(CSRC, s) for s in LIB_SOURCES]
    if force or _newer(LIB, srcs):
        # one object per translation unit, compiled in parallel, then linked
        os.makedirs(OBJ, exist_ok=True)
        gen = os.path.join(OBJ, "ctl_tiny_src.cpp")
        _embed_sources(gen)
        srcs = srcs + [gen]
        objs = [os.path.join(OBJ, os.path.basename(s) + ".o") for s in srcs]
        cmds = [["nvcc", *NVCC_FLAGS, "-c", src, "-o", obj] for src, obj in zip(srcs, objs)]
        jobs = max(1, min(len(cmds), os.cpu_count() or 1))
        with ThreadPoolExecutor(jobs) as ex:
            list(ex.map(lambda c: _run(c, verbose), cmds))
        _run(["nvcc", *ARCH, "-shared", "-o", LIB, *objs, "-ldl"], verbose)
    cli_srcs = [os.path.join(CSRC, s) for s in CLI_SOURCES]
    if force or _newer(CLI, cli_srcs + [LIB]):
        _run(["g++", "-O2", "-std=c++17", f"-I{INCLUDE}", "-o", CLI, *cli_srcs,
              f"-L{HERE}", "-lctl", "-Wl,-rpath,$ORIGIN"], verbose)


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
