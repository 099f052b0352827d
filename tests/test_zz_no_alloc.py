"""The allocation-free diagnostic sums (lbmc_macro_sums_noalloc).

Callers that cannot allocate device memory when they need the sums (their
own pool allocator already holds the device, a device-memory cap, or a time
loop that must not pay cudaMalloc's implicit synchronisation) use this entry
point instead of the handle's LBMC_REDUCE_DIAG path, which keeps per-block
scratch that lbmc_init allocated.  This test checks, through the C ABI, that
the new entry point gives the same sums as the existing path (lbmc_iterate
with LBMC_REDUCE_DIAG + lbmc_fetch(LBMC_FIELD_DIAG)) on two calls in a row,
within the tolerances of test_parity_gpu.test_diagnostics_fp64_sums, and that
it refuses sizes beyond its fixed scratch.  The file sorts last so that a
run stopping at the first failure has run everything else first.
"""
import numpy as np
import pytest

from cases import make_case

pytestmark = pytest.mark.gpu


def _sums_noalloc(lbmc, torch, rho, u):
    dev = torch.device("cuda", 0)
    r = torch.from_numpy(rho).to(dev)
    comps = [torch.from_numpy(np.ascontiguousarray(u[k])).to(dev) for k in range(3)]
    out = torch.full((5,), float("nan"), dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    st = lbmc.library().lbmc_macro_sums_noalloc(0, r.data_ptr(), comps[0].data_ptr(),
                                                 comps[1].data_ptr(), comps[2].data_ptr(),
                                                 r.numel(), out.data_ptr(), None)
    assert st == lbmc.OK, lbmc.library().lbmc_last_error()
    torch.cuda.synchronize()
    return out.cpu().numpy()


def _check(d, s):
    assert abs(s[0] - d.mass) <= 1e-12 * abs(d.mass)
    for k in range(3):
        assert abs(s[1 + k] - d.momentum[k]) <= 1e-9 * max(abs(d.mass) * 1e-6, abs(d.momentum[k]))
    assert abs(s[4] - d.kinetic_energy) <= 1e-10 * d.kinetic_energy


def test_noalloc_sums_match_handle_diagnostics(lbmc):
    import torch
    case = make_case("d3q15", (40, 36, 30), 2, True, solids=0.1, micro="zh", seed=21)
    with lbmc.Engine.from_case(case) as eng:
        for steps in (7, 13):  # two calls in a row, on different fields
            eng.iterate(steps, lbmc.STORE_MACROS | lbmc.REDUCE_DIAG | lbmc.SYNC)
            d = eng.diag()
            rho, u = eng.rho(), eng.u()
            s = _sums_noalloc(lbmc, torch, rho, u)
            _check(d, s)


def test_noalloc_rejects_sizes_beyond_scratch(lbmc):
    import torch
    x = torch.zeros(4, dtype=torch.float64, device="cuda")
    lib = lbmc.library()
    too_many = 134217728 + 1
    assert lib.lbmc_macro_sums_noalloc(0, x.data_ptr(), x.data_ptr(), None, None, too_many,
                                       x.data_ptr(), None) == lbmc.ERR_INVALID_ARG
    assert lib.lbmc_macro_sums_noalloc(0, x.data_ptr(), x.data_ptr(), None, None, 0,
                                       x.data_ptr(), None) == lbmc.ERR_INVALID_ARG
