"""Builds libwosgpu.so (sm_100a) in-tree with nvcc.

    python tetsuhiro-wos_b200/build.py [--force]

The shared object lands in tetsuhiro-wos_b200/lib/ next to the package, so it
travels with the source tree; the CUDA runtime is linked statically.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libwosgpu.so")
SOURCES = ["wos_kernels.cu", "wos_kernels_mix32.cu", "wos_kernels_mix64.cu", "wos_fast.cu", "wos_fast_cp.cu", "wos_schell.cu", "wos_aniso.cu", "wos_pipe.cu", "wos_elem.cu", "wos_api.cu", "wos_bpm.cu", "wos_batch.cu", "wos_design.cu", "wos_field_ops.cu", "wos_comm.cu", "wos_host.cu", "wos_ctx.cu", "wos_static.cu"]
HEADERS = ["wos_fft.cuh", "wos_kernels.cuh", "wos_kernels_dev.cuh", "wos_fast.cuh", "wos_fast_dev.cuh", "wos_fast_kern.cuh", "wos_pipe.cuh", "wos_api_internal.cuh"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-std=c++17", "-lineinfo",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
    "-I", os.path.join(ROOT, "include"),
]


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps.append(os.path.join(ROOT, "include", "wos_gpu.h"))
    deps.append(os.path.abspath(__file__))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not _stale():
        return LIB
    os.makedirs(LIBDIR, exist_ok=True)
    objs, procs = [], []
    for src in SOURCES:  # translation units compile in parallel
        obj = os.path.join(LIBDIR, src.replace(".cu", ".o"))
        cmd = [NVCC, *FLAGS, "-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        procs.append((subprocess.Popen(cmd), cmd))
        objs.append(obj)
    for p, cmd in procs:
        if p.wait() != 0:
            raise subprocess.CalledProcessError(p.returncode, cmd)
    tmp = LIB + ".tmp"
    cmd = [NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-cudart", "static",
           "-Xlinker", "--exclude-libs,ALL", *objs, "-ldl", "-o", tmp]
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    for o in objs:
        os.remove(o)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
