"""Builds the in-tree shared library ndg_cuda_b200/libndg_b200.so for sm_100a.

The library is plain nvcc output (no torch extension): host C++ compiled
without FMA contraction (the tables and topology must round as the
reference does), CUDA for sm_100a with line info for the profiler.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libndg_b200.so")
OBJ = os.path.join(HERE, "_build")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off", "-I", os.path.join(HERE, "..", "include")]
CUDA_FLAGS = ARCH + ["-lineinfo", "--expt-relaxed-constexpr", "-Xptxas", "-v"] if os.environ.get("NDG_PTXAS_VERBOSE") else ARCH + ["-lineinfo", "--expt-relaxed-constexpr"]

SOURCES = ["tables.cpp", "topology.cpp", "adapt.cpp", "adapt_h.cpp", "stage_kernels.cu", "general_kernels.cu", "estimator.cu", "context.cu",
           "adjoint_kernels.cu", "adjoint_host.cu", "stage_variants_fp64.cu", "stage_variants_fp32.cu", "stage_variants_tc64.cu", "stage_variants_tc32.cu",
           "delta_t_scratch.cu", "adapt_device.cu", "conforming_kernels.cu", "output.cu", "output_host.cu", "writer.cpp"]


def _compile(src: str) -> str:
    path = os.path.join(CSRC, src)
    obj = os.path.join(OBJ, src + ".o")
    if os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(path), *(os.path.getmtime(os.path.join(CSRC, h)) for h in os.listdir(CSRC) if h.endswith((".hpp", ".cuh")))) \
            and os.path.getmtime(obj) >= os.path.getmtime(os.path.join(HERE, "..", "include", "ndg_b200.h")):
        return obj
    flags = COMMON + (CUDA_FLAGS if src.endswith(".cu") else ["-x", "c++", "-Wno-deprecated-gpu-targets"])
    cmd = [NVCC] + flags + ["-c", path, "-o", obj]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n{res.stdout}\n{res.stderr}")
    if res.stderr.strip():
        sys.stderr.write(res.stderr)
    return obj


def build(force: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    if force:
        for f in os.listdir(OBJ):
            os.remove(os.path.join(OBJ, f))
    with ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        objs = list(ex.map(_compile, SOURCES))
    if not os.path.exists(OUT) or os.path.getmtime(OUT) < max(os.path.getmtime(o) for o in objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", OUT] + objs + ["-lcudart_static", "-lrt", "-ldl", "-lpthread"]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"link failed:\n{res.stdout}\n{res.stderr}")
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
