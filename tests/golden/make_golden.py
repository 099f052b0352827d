"""Generates tests/golden/*.npz from the reference's own step.

Runs the host-compiled reference (oracle/_ref, built from the reference
sources by oracle/build_ref.sh) on small seeded problems and stores inputs and
outputs.  The fixtures let the oracle restatement and the CUDA engine be
checked against the reference on machines where the reference tree is absent.

    python tests/golden/make_golden.py [NAME ...]

Each fixture holds: the case parameters, the input arrays, the populations
after ``nsteps`` steps (natural layout) and the stored rho/u of the last step.
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

from cases import make_case  # noqa: E402
from oracle.oracle import (COMPAT_AS_IS, COMPAT_MRTPOR_INPLACE, Reference,  # noqa: E402
                           reference_available)

NSTEPS = 7
SIZES = {"d2q9": (9, 6, 1), "d3q15": (5, 4, 3)}

# name: (lattice, collision_type, forcing, solids, partial, macro, micro, c_smag, variant
#        [, MRT rate on rho and j])
CASES = {
    "d2q9_bgk": ("d2q9", 0, False, 0.1, 0.0, None, None, 0.0, "asis"),
    "d2q9_bgk_guo": ("d2q9", 0, True, 0.1, 0.0, None, None, 0.0, "asis"),
    "d2q9_ntpor_guo": ("d2q9", 1, True, 0.1, 0.2, None, None, 0.0, "asis"),
    "d2q9_mrt": ("d2q9", 2, False, 0.1, 0.0, None, None, 0.0, "asis"),
    "d2q9_mrt_guo": ("d2q9", 2, True, 0.1, 0.0, "random", None, 0.0, "asis"),
    "d2q9_mrtpor_guo": ("d2q9", 3, True, 0.1, 0.2, None, None, 0.0, "asis"),
    "d2q9_bgk_zh": ("d2q9", 0, False, 0.1, 0.0, None, "zh", 0.0, "asis"),
    "d2q9_bgk_macro": ("d2q9", 0, True, 0.0, 0.0, "random", None, 0.0, "asis"),
    "d2q9_smag": ("d2q9", 0, True, 0.1, 0.0, None, None, 0.1, "patched"),
    "d2q9_ntpor_smag": ("d2q9", 1, False, 0.1, 0.2, None, None, 0.1, "patched"),
    "d3q15_bgk": ("d3q15", 0, False, 0.1, 0.0, None, None, 0.0, "asis"),
    "d3q15_bgk_guo": ("d3q15", 0, True, 0.1, 0.0, None, None, 0.0, "asis"),
    "d3q15_ntpor_guo": ("d3q15", 1, True, 0.1, 0.2, None, None, 0.0, "asis"),
    "d3q15_mrt_asis": ("d3q15", 2, True, 0.1, 0.0, None, None, 0.0, "asis"),
    "d3q15_mrt": ("d3q15", 2, False, 0.1, 0.0, None, None, 0.0, "patched"),
    "d3q15_mrt_guo": ("d3q15", 2, True, 0.1, 0.0, "random", None, 0.0, "patched"),
    "d3q15_mrtpor_guo": ("d3q15", 3, True, 0.1, 0.2, None, None, 0.0, "patched"),
    "d3q15_bgk_zh": ("d3q15", 0, False, 0.0, 0.0, None, "zh", 0.0, "asis"),
    "d3q15_mrt_zh": ("d3q15", 2, False, 0.1, 0.0, None, "zh", 0.0, "patched"),
    "d3q15_smag": ("d3q15", 0, True, 0.1, 0.0, None, None, 0.1, "patched"),
    # MRT with non-zero rates on the conserved moments (the general MRT kernel)
    "d2q9_mrt_cons": ("d2q9", 2, False, 0.1, 0.0, None, None, 0.0, "asis", 1.0),
    "d2q9_mrt_cons_guo": ("d2q9", 2, True, 0.1, 0.0, "random", None, 0.0, "asis", 1.0),
    "d2q9_mrtpor_cons_guo": ("d2q9", 3, True, 0.1, 0.2, None, None, 0.0, "asis", 1.1),
    "d3q15_mrt_cons_guo": ("d3q15", 2, True, 0.1, 0.0, "random", None, 0.0, "patched", 1.0),
    "d3q15_mrtpor_cons_guo": ("d3q15", 3, True, 0.1, 0.2, None, None, 0.0, "patched", 1.1),
    "d3q15_mrt_cons_zh": ("d3q15", 2, False, 0.1, 0.0, None, "zh", 0.0, "patched", 0.9),
}


def build_case(name: str, seed: int = 11):
    lat, ct, forcing, solids, partial, macro, micro, smag, variant, *cons = CASES[name]
    case = make_case(lat, SIZES[lat], ct, forcing, solids=solids, partial=partial,
                     macro=macro, micro=micro, c_smag=smag, seed=seed,
                     mrt_conserved=cons[0] if cons else 0.0)
    # The restatement reproduces a reference variant with these compat bits.
    case.compat = COMPAT_AS_IS if variant == "asis" else COMPAT_MRTPOR_INPLACE
    return case, variant


def main(names=None):
    """Writes the named fixtures (default: all)."""
    for name in names or CASES:
        case, variant = build_case(name)
        if not reference_available(case.lattice, variant):
            raise SystemExit("oracle/_ref is not built: run oracle/build_ref.sh first")
        ref = Reference(case, variant, nthreads=1)
        ref.run(NSTEPS, store_last=True)
        f = ref.f()
        rho, u = ref.macros()
        a = case.arrays()
        meta = dict(name=name, lattice=case.lattice, length=list(case.length), tau=case.tau,
                    tau_mrt=list(case.tau_mrt), c_smag=case.c_smag,
                    collision_type=case.collision_type, forcing=case.forcing,
                    macro_bc=case.macro_bc, micro_bc=case.micro_bc, compat=case.compat,
                    variant=variant, nsteps=NSTEPS)
        arrays = {k: v for k, v in a.items() if v is not None}
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), meta=json.dumps(meta),
                            out_f=f, out_rho=rho, out_u=u,
                            **{f"in_{k}": v for k, v in arrays.items()})
        print("wrote", name)


if __name__ == "__main__":
    main(sys.argv[1:])
