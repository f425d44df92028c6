"""Build the sm_100a shared library libfsb200.so in-tree with nvcc.

Every translation unit is compiled for sm_100a only, with --fmad=false so
the per-face/per-cell arithmetic keeps the reference's operation order (no
contraction into FMA) and the assembled coefficients match the CPU
restatement bit for bit.  The CUDA runtime is linked statically so the
library has no runtime dependency beyond the driver.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libfsb200.so")
SOURCES = ["fs_geometry.cu", "fs_simple.cu", "fs_turb.cu", "fs_energy.cu", "fs_time.cu", "fs_neutral.cu", "fs_solvers.cu", "fs_mg.cu", "fs_nn.cu", "fs_capi.cu"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "--fmad=false", "-lineinfo", "-Xcompiler", "-fPIC,-O2",
         "-I", os.path.join(HERE, "..", "include")] + os.environ.get("FSB200_NVCC_FLAGS", "").split()


def _stale(out: str, deps: list[str]) -> bool:
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, ptxas_info: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, h) for h in os.listdir(CSRC) if h.endswith((".cuh", ".h"))]
    headers.append(os.path.join(HERE, "..", "include", "fsb200.h"))
    objs = []
    for src in SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src.replace(".cu", ".o"))
        objs.append(o)
        if _stale(o, [s] + headers) or ptxas_info:
            cmd = [NVCC] + ARCH + FLAGS + (["-Xptxas", "-v"] if ptxas_info else []) + ["-c", s, "-o", o]
            if verbose:
                print(" ".join(cmd), flush=True)
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode != 0:
                sys.stderr.write(r.stdout + r.stderr)
                raise RuntimeError(f"nvcc failed on {src}")
            if ptxas_info:
                sys.stderr.write(r.stderr)
    if _stale(LIB, objs):
        cmd = [NVCC] + ARCH + ["-shared", "--cudart", "static", "-o", LIB] + objs + ["-lpthread", "-ldl", "-lrt"]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("nvcc link failed")
    return LIB


if __name__ == "__main__":
    build(verbose=True, ptxas_info="--ptxas" in sys.argv)
    print(LIB)
