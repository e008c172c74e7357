"""The prepare kernels' register and shared-memory budgets, from ptxas, as
the occupancy they are designed for needs them (CPU: nvcc cross-compiles).

On an SM of 64K registers and 228 KB of shared memory (1 KB reserved per
CTA), eight 128-thread YUV CTAs need at most 64 registers and 28,160 bytes
each, and ten 128-thread table CTAs at most 48 registers; a kernel that
grows past these silently loses a CTA per SM (the YUV kernel once held the
8-bit table it does not use and ran seven)."""

import os
import re
import shutil
import subprocess

import pytest

from vqm_b200 import build

SM_SHARED = 233472
CTA_RESERVED = 1024


def _ptxas_report(tmp_path):
    nvcc = build.NVCC if os.path.exists(build.NVCC) else shutil.which("nvcc")
    if nvcc is None:
        pytest.skip("nvcc not found")
    src = os.path.join(build.ROOT, "vqm_b200", "csrc", "ss2_prepare.cu")
    inc = os.path.join(os.path.dirname(os.path.dirname(nvcc)), "include")
    r = subprocess.run([nvcc, *build.ARCH, "-O3", "-std=c++17", "-fmad=false", "-Xptxas=-v",
                        "-I" + inc, "-c", src, "-o", str(tmp_path / "prepare.o")],
                       capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-3000:]
    kernels, name = {}, None
    for line in r.stderr.splitlines():
        m = re.search(r"Compiling entry function '\S*PrepareKernelILi(\d)ELb(\d)ELi(\d+)E", line)
        if m:
            name = tuple(int(g) for g in m.groups())
            continue
        if name is None:
            continue
        m = re.search(r"(\d+) bytes spill stores", line)
        if m:
            kernels.setdefault(name, {})["spill"] = int(m.group(1))
        m = re.search(r"Used (\d+) registers.*?(\d+) bytes smem", line)
        if m:
            kernels.setdefault(name, {}).update(regs=int(m.group(1)), smem=int(m.group(2)))
            name = None
    return kernels


def test_prepare_kernels_fit_their_occupancy(tmp_path):
    k = _ptxas_report(tmp_path)
    for half in (0, 1):
        yuv = k[(1, half, 128)]
        assert yuv["regs"] * 128 * 8 <= 65536 and yuv["spill"] == 0, yuv
        assert 8 * (yuv["smem"] + CTA_RESERVED) <= SM_SHARED, yuv
        table = k[(0, half, 128)]
        assert table["regs"] * 128 * 10 <= 65536, table
        assert 10 * (table["smem"] + CTA_RESERVED) <= SM_SHARED, table
