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


def _check_against_torch(torch, rho, u, s):
    """FP64 sums of the same device arrays by torch (tolerance relative to
    the sum of magnitudes, 1e-12)."""
    terms = [rho, rho * u[0], rho * u[1], rho * u[2], 0.5 * rho * (u * u).sum(0)]
    for k, t in enumerate(terms):
        ref = float(t.sum())
        scale = float(t.abs().sum())
        assert abs(s[k] - ref) <= 1e-12 * scale, (k, s[k], ref)


def _device_fields(torch, n, seed):
    g = torch.Generator(device="cuda").manual_seed(seed)
    rho = 1 + 0.01 * torch.randn(n, dtype=torch.float64, device="cuda", generator=g)
    u = 0.05 * torch.randn((3, n), dtype=torch.float64, device="cuda", generator=g)
    return rho, u


def _call(lbmc, torch, rho, u):
    out = torch.full((5,), float("nan"), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    st = lbmc.library().lbmc_macro_sums_noalloc(0, rho.data_ptr(), u[0].data_ptr(), u[1].data_ptr(),
                                                 u[2].data_ptr(), rho.numel(), out.data_ptr(), None)
    assert st == lbmc.OK, lbmc.library().lbmc_last_error()
    torch.cuda.synchronize()
    return out.cpu().numpy()


def test_noalloc_sums_large_sizes_then_small(lbmc):
    """More blocks than the finalize kernel's threads (a ragged 5,000,003
    nodes: 306 blocks), the largest accepted size (2^27 nodes: every slot of
    the fixed scratch), then a small call that must not read the partials
    the large calls left behind."""
    import torch
    for n, seed in ((5_000_003, 1), (134_217_728, 2), (1000, 3)):
        rho, u = _device_fields(torch, n, seed)
        s = _call(lbmc, torch, rho, u)
        _check_against_torch(torch, rho, u, s)
        del rho, u
        torch.cuda.empty_cache()


def test_noalloc_reports_its_errors(lbmc):
    """Rejected calls set a message of their own (not one left over from an
    earlier call)."""
    lib = lbmc.library()
    assert lib.lbmc_macro_sums_noalloc(0, None, None, None, None, 10, None, None) == lbmc.ERR_INVALID_ARG
    assert b"NULL" in lib.lbmc_last_error()
    import torch
    x = torch.zeros(4, dtype=torch.float64, device="cuda")
    assert lib.lbmc_macro_sums_noalloc(0, x.data_ptr(), x.data_ptr(), None, None, 1 << 28,
                                       x.data_ptr(), None) == lbmc.ERR_INVALID_ARG
    assert b"exceeds" in lib.lbmc_last_error()
