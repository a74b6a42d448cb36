"""Builds libncsim_cuda.so in-tree for sm_100a (nvcc, no JIT cache).

Usage: ``python -m ncsim_b200.build`` (incremental; ``--force`` rebuilds).
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(PKG, "csrc")
OBJ = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libncsim_cuda.so")
WORKLOADS_LIB = os.path.join(PKG, "libncsim_workloads.so")

SOURCES = [
    "csrc/capi_state.cu",
    "csrc/kernels_plain.cu",
    "csrc/wide.cu",
    "csrc/plain_pass.cu",
    "csrc/fused.cu",
    "csrc/fused_plan.cpp",
    "csrc/batch.cu",
    "csrc/batch_plan.cpp",
    "csrc/sparse.cu",
    "csrc/sparse_wide.cu",
    "csrc/frames.cu",
    "csrc/frames_plan.cpp",
    "csrc/host/ir.cpp",
    "csrc/host/runtime.cpp",
]
# the seeded synthetic workloads of the benchmark and the tests: a second
# library on top of the engine, outside the drop-in interface
WORKLOAD_SOURCES = ["csrc/workloads/workloads.cpp"]
HEADERS = [
    "csrc/engine.cuh",
    "csrc/sparse_common.cuh",
    "csrc/host_math.hpp",
    "csrc/fused_plan.hpp",
    "csrc/batch_plan.hpp",
    "csrc/frames_plan.hpp",
    "csrc/host/ir.hpp",
    "csrc/host/rng.hpp",
    "../include/ncsim_cuda.h",
    "../include/ncsim_workloads.h",
]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ARCH + [
    "-O3",
    "-lineinfo",
    "-std=c++17",
    "--expt-relaxed-constexpr",
    "-Xcompiler",
    "-fPIC,-O3",
    "-Xcudafe",
    "--diag_suppress=177",
]


def _nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


CUDA_INCLUDE = "/usr/local/cuda/include"


def _newer(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False, ptxas_info: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    nvcc = _nvcc()
    env = dict(os.environ)
    env.pop("CXX", None)  # the host compiler is nvcc's default (the system g++)
    headers = [os.path.join(PKG, h) for h in HEADERS]
    objs, wobjs = [], []
    procs = []
    for src in SOURCES + WORKLOAD_SOURCES:
        path = os.path.join(PKG, src)
        obj = os.path.join(OBJ, src.replace("/", "_") + ".o")
        (wobjs if src in WORKLOAD_SOURCES else objs).append(obj)
        if force or _newer(obj, [path] + headers):
            if src in WORKLOAD_SOURCES:  # host code only: compiled by the host compiler, no device image
                cmd = ["g++", "-std=c++17", "-O3", "-fPIC", "-I" + CUDA_INCLUDE, "-c", path, "-o", obj]
            else:
                cmd = [nvcc] + NVFLAGS + ["-x", "cu", "-c", path, "-o", obj]
            if ptxas_info:
                cmd += ["-Xptxas", "-v"]
            if verbose:
                print(" ".join(cmd), flush=True)
            procs.append((src, subprocess.Popen(cmd, env=env, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
    failed = []
    for src, p in procs:
        out, _ = p.communicate()
        text = out.decode(errors="replace")
        if p.returncode != 0:
            failed.append((src, text))
        elif verbose and text.strip():
            print(text)
    if failed:
        for src, text in failed:
            sys.stderr.write(f"--- {src}\n{text}\n")
        raise RuntimeError("nvcc failed for " + ", ".join(s for s, _ in failed))
    if force or _newer(LIB, objs):
        cmd = [nvcc] + ARCH + ["-shared", "-o", LIB] + objs + ["-cudart", "static", "-lpthread",
                                                              "-Xlinker", "-soname=libncsim_cuda.so"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True, env=env)
    if force or _newer(WORKLOADS_LIB, wobjs + [LIB]):
        # resolves the engine's symbols from libncsim_cuda.so beside it (no CUDA runtime of its own)
        cmd = ["g++", "-shared", "-o", WORKLOADS_LIB] + wobjs + ["-L" + PKG, "-lncsim_cuda", "-Wl,-rpath,$ORIGIN"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True, env=env)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv, ptxas_info="--ptxas" in sys.argv)
    print(LIB)
