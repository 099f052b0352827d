"""GPU parity of the general MRT kernel: non-zero relaxation rates on the
conserved moments (rho, j), as a TauMRT input line sets them
(LBM-C/infile_reader.cu:63-76 reads the rates; LBM-C/collision.cu:192-421
relaxes every moment with its own rate).

The engine compiles two MRT collisions: one that skips the conserved
moments when their rates are zero (the porous benchmark's rates) and the
general one these tests reach.  Each case runs 100 steps through the C ABI
and is compared with the reference's own step (host-compiled, patched build;
the FP64 restatement where that library is absent) in every streaming
layout and both step kernels.  Error measure and bounds as in
test_parity_gpu: err(X) = max|X_gpu - X_ref| / max|X_ref|, <= 1e-5 with FP32
storage, <= 1e-10 with FP64 storage.
"""
import numpy as np
import pytest

from cases import make_case
from oracle.oracle import COMPAT_MRTPOR_INPLACE, Reference, Restatement, reference_available

pytestmark = pytest.mark.gpu

TOL = {"f64": 1e-10, "f32": 1e-5}
STEPS = 100

COMBOS = [(lat, ct, forcing, bc) for lat in ("d2q9", "d3q15") for ct in (2, 3)
          for forcing in (False, True) for bc in (None, "random", "zh")]

# layout: (streaming, kernel, D2Q9 length, D3Q15 length).  Rows of 40 / 24
# elements are whole 16-byte granules, which the bulk-copy kernel needs;
# Lx = 64 selects the tiled AA layout.
LAYOUTS = {
    "shift": ("shift", "direct", (37, 21, 1), (19, 11, 9)),
    "shift_pipelined": ("shift", "pipelined", (40, 21, 1), (24, 11, 9)),
    "aa": ("aa", "direct", (37, 21, 1), (19, 11, 9)),
    "aa_tiled": ("aa", "direct", (64, 21, 1), (64, 7, 6)),
}


def err(a, b):
    a, b = np.asarray(a), np.asarray(b)
    scale = np.abs(b).max()
    return float(np.abs(a - b).max() / (scale if scale > 0 else 1.0))


_REF_CACHE = {}


def reference_state(lat, ct, forcing, bc, length):
    key = (lat, ct, forcing, bc, length)
    if key not in _REF_CACHE:
        case = make_case(lat, length, ct, forcing, solids=0.08, partial=0.15 if ct == 3 else 0.0,
                         macro="random" if bc == "random" else None,
                         micro="zh" if bc == "zh" else None, seed=41 + ct, mrt_conserved=1.05)
        # The patched reference keeps the MRTPOR in-place blend (it fixes
        # only the D3Q15 M_inv, -7/3 and +z Zou-He defects); the engine
        # reproduces it with the compat bit.
        case.compat = COMPAT_MRTPOR_INPLACE
        if reference_available(lat, "patched"):
            ref = Reference(case, "patched")
        else:
            ref = Restatement(case)
        ref.run(STEPS)
        rho, u = ref.macros()
        _REF_CACHE[key] = (case, ref.f(), rho, u)
    return _REF_CACHE[key]


@pytest.mark.parametrize("layout", list(LAYOUTS))
@pytest.mark.parametrize("lat,ct,forcing,bc", COMBOS)
def test_conserved_rate_mrt_matches_reference(lbmc, lat, ct, forcing, bc, layout):
    streaming, kernel, len2, len3 = LAYOUTS[layout]
    case, f_ref, rho_ref, u_ref = reference_state(lat, ct, forcing, bc, len2 if lat == "d2q9" else len3)
    assert any(case.tau_mrt[k] != 0 for k in (0, 3, 5)), "the general MRT kernel must run"
    kw = dict(streaming=lbmc.STREAM_AA if streaming == "aa" else lbmc.STREAM_SHIFT,
              kernel=lbmc.KERNEL_PIPELINED if kernel == "pipelined" else lbmc.KERNEL_DIRECT)
    for storage in ("f64", "f32"):
        with lbmc.Engine.from_case(case, storage=lbmc.STORAGE_IDS[storage], **kw) as eng:
            eng.iterate(STEPS, lbmc.STORE_MACROS | lbmc.SYNC)
            f, rho, u = eng.f(), eng.rho(), eng.u()
        tol = TOL[storage]
        assert err(f, f_ref) <= tol, storage
        assert err(rho, rho_ref) <= tol, storage
        assert err(u, u_ref) <= tol, storage


@pytest.mark.parametrize("lat", ["d2q9", "d3q15"])
def test_conserved_rates_change_the_forced_result(lbmc, lat):
    """With Guo forcing, j - rho u = -F/2 is non-zero, so a rate on j changes
    the result: the general kernel is not silently the zero-rate one."""
    length = (37, 21, 1) if lat == "d2q9" else (19, 11, 9)
    out = []
    for cons in (0.0, 1.05):
        case = make_case(lat, length, 2, True, solids=0.08, seed=43, mrt_conserved=cons)
        with lbmc.Engine.from_case(case, storage=lbmc.F64) as eng:
            eng.iterate(20, lbmc.STORE_MACROS | lbmc.SYNC)
            out.append(eng.u())
    assert err(out[1], out[0]) > 1e-6
