"""Build the CUDA engine (libsmfg.so) in-tree for sm_100a.

    python -m opt_solver_b200.build

The library is a plain C ABI (include/smfg.h) over the CUDA runtime; it does
not link against PyTorch. ``--fmad=false``: no multiply-add is contracted
implicitly; the kernels call fma() where smf's arithmetic fuses and
__dmul_rn / __dadd_rn / __dsub_rn where it does not.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libsmfg.so")
SOURCES = ["smfg_engine.cu", "smfg_analyse.cpp", "smfg_scaling.cpp", "smfg_mlp.cu"]
DEPS = ["smfg_front.cuh", "smfg_kernels.cuh", "smfg_internal.cuh", "smfg_tc.cuh"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def flags(extra=()):
    return [
        "-O3", "-std=c++17", "--fmad=false", "-lineinfo",
        "-gencode", "arch=compute_100a,code=sm_100a",
        "-Xcompiler", "-fPIC,-fvisibility=hidden", "-shared",
        "-I" + os.path.join(ROOT, "include"),
        *extra,
    ]


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    srcs = [os.path.join(CSRC, s) for s in SOURCES + DEPS] + [os.path.join(ROOT, "include", "smfg.h")]
    return any(os.path.getmtime(s) > t for s in srcs if os.path.exists(s))


def build(force: bool = False, verbose: bool = False, ptxas_info: bool = False) -> str:
    if not force and not needs_build():
        return LIB
    extra = ["-Xptxas", "-v"] if ptxas_info else []
    cmd = [nvcc(), *flags(extra), "-o", LIB + ".tmp", *[os.path.join(CSRC, s) for s in SOURCES],
           "-lcudart"]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc failed")
    if verbose or ptxas_info:
        sys.stderr.write(r.stderr)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, ptxas_info="--ptxas" in sys.argv)
    print(LIB)
