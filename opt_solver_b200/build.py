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
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libsmfg.so")
SOURCES = ["smfg_engine.cu", "smfg_aptp.cu", "smfg_analyse.cpp", "smfg_scaling.cpp", "smfg_mlp.cu"]
DEPS = ["smfg_front.cuh", "smfg_kernels.cuh", "smfg_internal.cuh", "smfg_tc.cuh", "smfg_aptp.cuh",
        "smfg_aptp_host.h"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def flags(extra=()):
    return [
        "-O3", "-std=c++17", "--fmad=false", "-lineinfo",
        "-gencode", "arch=compute_100a,code=sm_100a",
        "-Xcompiler", "-fPIC,-fvisibility=hidden",
        "-I" + os.path.join(ROOT, "include"),
        *extra,
    ]


def _inputs():
    return [os.path.join(CSRC, s) for s in DEPS] + [os.path.join(ROOT, "include", "smfg.h"), __file__]


def _obj(src: str) -> str:
    return os.path.join(OBJ, src + ".o")


def _stale(target: str, srcs) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in srcs if os.path.exists(s))


def needs_build() -> bool:
    return _stale(LIB, [os.path.join(CSRC, s) for s in SOURCES] + _inputs())


def build(force: bool = False, verbose: bool = False, ptxas_info: bool = False) -> str:
    """Compile each source to an object (in parallel, only those older than
    their inputs unless force), then link the shared library."""
    if not force and not needs_build():
        return LIB
    os.makedirs(OBJ, exist_ok=True)
    extra = ["-Xptxas", "-v"] if ptxas_info else []
    procs = []
    for src in SOURCES:
        obj = _obj(src)
        if not force and not _stale(obj, [os.path.join(CSRC, src)] + _inputs()):
            continue
        cmd = [nvcc(), *flags(extra), "-c", os.path.join(CSRC, src), "-o", obj + ".tmp"]
        if verbose:
            print(" ".join(cmd), flush=True)
        procs.append((obj, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True)))
    failed = False
    for obj, pr in procs:
        out, err = pr.communicate()
        if pr.returncode != 0:
            sys.stderr.write(out + err)
            failed = True
        else:
            if verbose or ptxas_info:
                sys.stderr.write(err)
            os.replace(obj + ".tmp", obj)
    if failed:
        raise RuntimeError("nvcc failed")
    cmd = [nvcc(), "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", LIB + ".tmp",
           *[_obj(s) for s in SOURCES], "-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("link failed")
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, ptxas_info="--ptxas" in sys.argv)
    print(LIB)
