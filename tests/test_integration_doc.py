"""The C binding example in INTEGRATION.md (section 1) is what a maintainer
copies into LBM-C's host code (LBM-C/index.cu's setup / iterate / output
functions), so it must compile and link against include/lbmc.h and
liblbmc.so as written.  LBM-C's own Domain and DomainConstant types
(LBM-C/data_types.cuh:13-43) are stood in for by the fields the example
reads, with the same names and types; DIM/Q select D3Q15 as LBM-C's
macros.cu does.  Compile and
link only: nothing runs, so no GPU is needed."""
import os
import re
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PRELUDE = """#include <stdio.h>
#include <stdlib.h>
#include <stdbool.h>
#define DIM 3
#define Q 15
typedef struct { int length[DIM]; double tau, tau_mrt[Q], c_smag; int collision_type;
                 bool forcing, macro_bc, micro_bc; } DomainConstant;
typedef struct { double *geometry, **force, **u, *rho; int *macro_bc, *micro_bc; } Domain;
"""

MAIN = """
int main(void)
{
    /* Referenced, not called: linking proves every symbol resolves. */
    void *fns[] = {(void *)setup_lbmc, (void *)iterate_lbmc, (void *)output_macros_lbmc,
                   (void *)kinetic_energy_lbmc};
    return fns[0] == NULL;
}
"""


def _snippet():
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    section = text.split("## 1.", 1)[1].split("\n## ", 1)[0]
    blocks = re.findall(r"```c\n(.*?)```", section, re.S)
    assert blocks, "no C block in section 1"
    return blocks[0]


def test_c_binding_example_compiles_and_links(tmp_path):
    cc = shutil.which("gcc") or shutil.which("cc")
    lib = os.path.join(ROOT, "lbm-c_b200", "liblbmc.so")
    if cc is None:
        pytest.skip("no C compiler")
    if not os.path.exists(lib):
        pytest.skip("liblbmc.so not built")
    src = tmp_path / "binding.c"
    src.write_text(PRELUDE + _snippet() + MAIN)
    out = tmp_path / "binding"
    run = subprocess.run(
        [cc, "-std=c99", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"), str(src),
         "-L", os.path.dirname(lib), "-llbmc", "-Wl,-rpath," + os.path.dirname(lib), "-o", str(out)],
        capture_output=True, text=True, timeout=300)
    assert run.returncode == 0, run.stderr[-4000:]
