"""Streaming maps of the direct step kernel, checked on the CPU.

Compiles tests/layout_check.cu, which includes the kernel header and runs
the same read/write pointer functions, site set-up and cold-kernel slot map
that the step kernel uses, over every node and population of small D2Q9 and
D3Q15 domains for the shift layout (LBM-C/solver.cu:82-94), the AA layout
and the tiled AA layout: range, one read per element per step, in-place
writes, streaming to the neighbour at the next step, and agreement with the
fetch/upload map.
"""
import os
import shutil
import subprocess
from pathlib import Path

import pytest

HERE = Path(__file__).resolve().parent


def _nvcc():
    found = shutil.which("nvcc")
    if found:
        return found
    default = "/usr/local/cuda/bin/nvcc"
    return default if os.path.exists(default) else None


def test_streaming_maps(tmp_path):
    nvcc = _nvcc()
    if nvcc is None:
        pytest.skip("nvcc not found")
    exe = tmp_path / "layout_check"
    build = subprocess.run(
        [nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-std=c++17", "-O1",
         str(HERE / "layout_check.cu"), "-o", str(exe)],
        capture_output=True, text=True, timeout=600)
    assert build.returncode == 0, build.stderr[-4000:]
    run = subprocess.run([str(exe)], capture_output=True, text=True, timeout=600)
    assert run.returncode == 0, run.stdout[-4000:]
    assert run.stdout.startswith("OK"), run.stdout
