"""The C binding example (tests/c/lbmc_binding.c, quoted in the integration
guide) is what a maintainer copies into LBM-C's host code (LBM-C/index.cu's
setup / iterate / output functions), so it must compile and link against
include/lbmc.h and liblbmc.so as written.  Compile and link only: nothing
runs, so no GPU is needed."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "c", "lbmc_binding.c")


def test_c_binding_example_compiles_and_links(tmp_path):
    cc = shutil.which("gcc") or shutil.which("cc")
    lib = os.path.join(ROOT, "lbm-c_b200", "liblbmc.so")
    if cc is None:
        pytest.skip("no C compiler")
    if not os.path.exists(lib):
        pytest.skip("liblbmc.so not built")
    out = tmp_path / "binding"
    run = subprocess.run(
        [cc, "-std=c99", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"), SRC,
         "-L", os.path.dirname(lib), "-llbmc", "-Wl,-rpath," + os.path.dirname(lib), "-o", str(out)],
        capture_output=True, text=True, timeout=300)
    assert run.returncode == 0, run.stderr[-4000:]
