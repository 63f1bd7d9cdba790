"""Swizzled shared-memory layouts of the multi-pass and macro-path kernels,
checked on the CPU.

tests/cpp/exchange_layout_check.cu includes the kernel headers and calls
their own index functions: pass_xidx on the positions every shared-memory
access of the 512- and 1024-point passes touches (both precisions and both
pass schemes), and keep_idx on the macro path's segment tiles (micro orders
8-12). It checks that each layout is a bijection, that the pass kernel's
split of a position into a thread part and a compile-time part gives the
same index, and that no access has a bank conflict. As a control, the padded
layout that the passes used before must show conflicts. Host code only: nvcc
compiles it for sm_100a, but nothing runs on a GPU.
"""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_swizzled_layouts_are_bijective_and_conflict_free(tmp_path):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not available")
    exe = str(tmp_path / "exchange_layout_check")
    cmd = [nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-std=c++20", "-O1", "--expt-relaxed-constexpr",
           "-I", os.path.join(ROOT, "zldsp_fft_b200", "csrc"), "-I", os.path.join(ROOT, "include"),
           "-x", "cu", os.path.join(ROOT, "tests", "cpp", "exchange_layout_check.cu"), "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    lines = r.stdout.splitlines()
    assert sum(1 for line in lines if line.endswith("(0 extra wavefronts)") and ": ok" in line) == 23, r.stdout
    assert any(line.startswith("control:") and "(detected)" in line for line in lines), r.stdout
