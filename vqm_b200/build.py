"""Builds libvqm_ss2.so in place: the sm_100a kernels, the host runtime and
the C ABI declared in include/vqm_cu_ss2.h.

    python -m vqm_b200.build            # incremental
    python -m vqm_b200.build --force

Device code is compiled with -fmad=false: every fused multiply-add in the
kernels is written out (__fmaf_rn), so the rounding is fixed by the source.
"""

from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(ROOT, "_build")
LIB = os.path.join(PKG, "libvqm_ss2.so")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
CXX = os.environ.get("CXX", "g++")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

CUDA_SOURCES = ["ss2_prepare.cu", "ss2_blur.cu", "ss2_runtime.cu",
                "ss2_noalloc.cu"]
HOST_SOURCES = ["ss2_host.cc", "ss2_server.cc"]
HEADERS = ["ss2_device.cuh", "ss2_decode.cuh", "ss2_detmath.h", "ss2_kernels.h", "ss2_host.h",
           "ss2_layout.h", "ss2_detmath_tables.h"]


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd: list[str]) -> None:
    print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build(force: bool = False, verbose_ptxas: bool = False) -> str:
    """Compiles what changed and links the shared library; returns its path."""
    if not os.path.exists(NVCC) and shutil.which("nvcc") is None:
        raise RuntimeError("nvcc not found: the CUDA extension cannot be built")
    nvcc = NVCC if os.path.exists(NVCC) else shutil.which("nvcc")
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, h) for h in HEADERS]
    headers.append(os.path.join(ROOT, "include", "vqm_cu_ss2.h"))
    objects = []
    for src in CUDA_SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(BUILD, src + ".o")
        objects.append(obj)
        if force or _stale(obj, [path] + headers):
            cmd = [nvcc, *ARCH, "-lineinfo", "-O3", "-std=c++17", "-fmad=false",
                   "-Xcompiler", "-fPIC,-ffp-contract=off", "-c", path, "-o", obj]
            if verbose_ptxas:
                cmd.insert(1, "-Xptxas=-v")
            _run(cmd)
    for src in HOST_SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(BUILD, src + ".o")
        objects.append(obj)
        if force or _stale(obj, [path] + headers):
            cuda_inc = os.path.join(os.path.dirname(os.path.dirname(nvcc)), "include")
            _run([CXX, "-O2", "-std=c++17", "-fPIC", "-ffp-contract=off",
                  "-fno-fast-math", "-I" + cuda_inc, "-c", path, "-o", obj])
    if force or _stale(LIB, objects):
        _run([nvcc, *ARCH, "-shared", "-o", LIB, *objects, "-lcudart"])
    return LIB


def main(argv: list[str] | None = None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--ptxas", action="store_true", help="print -Xptxas -v")
    args = ap.parse_args(argv)
    build(force=args.force, verbose_ptxas=args.ptxas)
    return 0


if __name__ == "__main__":
    sys.exit(main())
