"""C-ABI library checks that need no GPU: the in-tree liblbmc.so loads,
exports every function include/lbmc.h declares, validates its inputs the way
the reference's codes require, and reports a missing device as a status."""
import ctypes

import numpy as np
import pytest

from cases import make_case
from oracle.oracle import Restatement


def test_library_exports_every_header_function(lbmc):
    lib = lbmc.library()
    names = lbmc.header_functions()
    assert "lbmc_init" in names and "lbmc_iterate" in names and "lbmc_fetch" in names
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_status_strings(lbmc):
    lib = lbmc.library()
    for s in range(10):
        assert lib.lbmc_status_string(s)


@pytest.mark.parametrize("lat", ["d2q9", "d3q15"])
def test_lattice_tables_match_oracle(lbmc, lat):
    q, dim = (9, 2) if lat == "d2q9" else (15, 3)
    e = np.zeros((dim, q), np.int32)
    w = np.zeros(q)
    opp = np.zeros(q, np.int32)
    m = np.zeros((q, q), np.int32)
    lbmc.check(lbmc.library().lbmc_lattice_tables(
        lbmc.LATTICE_IDS[lat], e.ctypes.data, w.ctypes.data, opp.ctypes.data, m.ctypes.data))
    e2, w2, opp2, M2, _ = Restatement(make_case(lat, (3, 3, 3))).tables()
    np.testing.assert_array_equal(e, e2)
    np.testing.assert_allclose(w, w2, rtol=1e-15)
    np.testing.assert_array_equal(opp, opp2)
    np.testing.assert_array_equal(m, M2)


def _validate(lbmc, case, **kw):
    a = case.arrays()
    cfg = lbmc.make_config(case.lattice, case.length, tau=case.tau, tau_mrt=case.tau_mrt,
                           collision_type=case.collision_type, forcing=case.forcing,
                           macro_bc=case.macro_bc, micro_bc=case.micro_bc, **kw)
    dom, keep = lbmc.make_domain(case.n, case.dim, case.q, a["geometry"], a["force"],
                                 a["macro"], a["micro"], a["u"], a["rho"], a["f0"])
    return lbmc.library().lbmc_validate(ctypes.byref(cfg), ctypes.byref(dom)), cfg, dom, keep


def test_validate_accepts_good_case(lbmc):
    case = make_case("d3q15", (6, 5, 4), 2, True, solids=0.1, micro="zh")
    st, *_ = _validate(lbmc, case)
    assert st == lbmc.OK


def test_validate_rejects_null_d2q9_micro_codes(lbmc):
    """micro_bc.cuh:7-8 leaves D2Q9 codes 3 and 4 NULL; the engine refuses them."""
    case = make_case("d2q9", (8, 6, 1), micro="zh")
    case.micro = case.micro.copy()
    case.micro[9] = 3
    st, *_ = _validate(lbmc, case)
    assert st == lbmc.ERR_INVALID_ARG
    assert b"undefined for D2Q9" in lbmc.library().lbmc_last_error()


@pytest.mark.parametrize("field,value", [("macro", 16), ("micro", 13), ("macro", -1)])
def test_validate_rejects_out_of_range_codes(lbmc, field, value):
    case = make_case("d3q15", (5, 4, 3), macro="random", micro="zh")
    arr = getattr(case, field).copy()
    arr[7] = value
    setattr(case, field, arr)
    st, *_ = _validate(lbmc, case)
    assert st == lbmc.ERR_INVALID_ARG


def test_validate_rejects_bad_parameters(lbmc):
    case = make_case("d2q9", (8, 6, 1))
    assert _validate(lbmc, case, storage=7)[0] == lbmc.ERR_INVALID_ARG
    assert _validate(lbmc, case, compat=1 << 9)[0] == lbmc.ERR_INVALID_ARG
    bad = make_case("d2q9", (8, 6, 1))
    bad.tau = -1.0
    assert _validate(lbmc, bad)[0] == lbmc.ERR_INVALID_ARG
    smag_mrt = make_case("d3q15", (4, 4, 4), 2, c_smag=0.1)
    assert _validate(lbmc, smag_mrt, c_smag=0.1)[0] == lbmc.ERR_UNSUPPORTED


def test_validate_fp16_scale_is_a_power_of_two(lbmc):
    """FP16 stores (f - w) * scale; the load multiplies back by 1/scale in
    one fused FP16 x FP16 -> FP32 step, exact only for powers of two."""
    case = make_case("d2q9", (8, 6, 1))
    for bad in (1000.0, 3.0, 2.0 ** 15, 2.0 ** -16):
        assert _validate(lbmc, case, storage=lbmc.F16, storage_scale=bad)[0] == lbmc.ERR_INVALID_ARG
    for ok in (0.0, 1.0, 1024.0, 2048.0, 2.0 ** -15, 2.0 ** 14):
        assert _validate(lbmc, case, storage=lbmc.F16, storage_scale=ok)[0] == lbmc.OK
    assert _validate(lbmc, case, storage=lbmc.F32, storage_scale=1000.0)[0] == lbmc.OK
    with pytest.raises(lbmc.LbmcError) as ei:
        lbmc.Batch([np.zeros((4, 4))], storage=lbmc.F16, storage_scale=1000.0)
    assert ei.value.status == lbmc.ERR_INVALID_ARG


def test_classify_packs_codes(lbmc):
    case = make_case("d3q15", (6, 5, 4), 3, solids=0.1, partial=0.2, micro="zh")
    st, cfg, dom, keep = _validate(lbmc, case)
    assert st == lbmc.OK
    cls = np.zeros(case.n, np.uint8)
    table = np.zeros(256, np.uint16)
    ncls = ctypes.c_int()
    lbmc.check(lbmc.library().lbmc_classify(ctypes.byref(cfg), ctypes.byref(dom),
                                            cls.ctypes.data, table.ctypes.data,
                                            ctypes.byref(ncls)))
    B = case.geometry
    assert np.all((cls == 1) == (B >= 1))
    for k in range(case.n):
        if B[k] >= 1:
            continue
        entry = int(table[cls[k]]) if cls[k] >= 2 else 0
        assert entry & 0xF == case.macro[k]
        assert (entry >> 4) & 0xF == case.micro[k]
        assert bool(entry & 0x100) == (B[k] != 0)


def test_init_without_device_reports_status(lbmc):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    case = make_case("d2q9", (8, 6, 1))
    with pytest.raises(lbmc.LbmcError) as ei:
        lbmc.Engine.from_case(case)
    assert ei.value.status == lbmc.ERR_NO_DEVICE


@pytest.mark.parametrize("length,status", [
    ((2048, 1024, 1025), "ERR_UNSUPPORTED"),   # over 2^31 nodes: 32-bit slot offsets
    ((8, 70000, 2), "ERR_UNSUPPORTED"),        # Ly over 65535 grid rows
    ((0, 4, 4), "ERR_INVALID_ARG"), ((4, -1, 4), "ERR_INVALID_ARG")])
def test_validate_rejects_sizes(lbmc, length, status):
    """Sizes are checked before any per-node work: no arrays are read."""
    cfg = lbmc.make_config("d3q15", length, tau=0.8)
    dom = lbmc.Domain()
    st = lbmc.library().lbmc_validate(ctypes.byref(cfg), ctypes.byref(dom))
    assert st == getattr(lbmc, status)


def test_fetch_out_arrays_are_checked(lbmc):
    """Engine.rho(out=...) / u(out=...) fill caller arrays of the exact
    shape and type only (lbmc_fetch writes FP64 node-order arrays)."""
    from lbmc import _checked_out
    ok = np.zeros((3, 10))
    assert _checked_out(ok, (3, 10)) is ok
    for bad in (np.zeros((3, 10), np.float32), np.zeros((10, 3)), np.zeros((3, 20))[:, ::2], [0.0] * 30):
        with pytest.raises(ValueError):
            _checked_out(bad, (3, 10))
