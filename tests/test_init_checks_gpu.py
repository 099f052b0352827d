"""lbmc_init checks the per-node inputs (porosity, MacroBC and MicroBC codes,
the fields a code needs) in the same pass over the arrays that packs the
node classes, on the host's cores while rho and u upload.  It must reject
what lbmc_validate rejects, with the same status and message, and name the
first bad node in node order also when several host threads scan the
domain.  A handle made after a rejected one must work."""
import ctypes

import numpy as np
import pytest

from cases import make_case

pytestmark = pytest.mark.gpu


def _validate(lbmc, case):
    a = case.arrays()
    cfg = lbmc.make_config(case.lattice, case.length, tau=case.tau, tau_mrt=case.tau_mrt,
                           collision_type=case.collision_type, forcing=case.forcing,
                           macro_bc=case.macro_bc, micro_bc=case.micro_bc)
    dom, keep = lbmc.make_domain(case.n, case.dim, case.q, a["geometry"], a["force"],
                                 a["macro"], a["micro"], a["u"], a["rho"], a["f0"])
    lib = lbmc.library()
    st = lib.lbmc_validate(ctypes.byref(cfg), ctypes.byref(dom))
    del keep
    return st, lib.lbmc_last_error().decode()


def _init_error(lbmc, case):
    with pytest.raises(lbmc.LbmcError) as ei:
        lbmc.Engine.from_case(case)
    return ei.value.status, lbmc.library().lbmc_last_error().decode()


def _set(case, field, k, value):
    arr = getattr(case, field).copy()
    arr[k] = value
    setattr(case, field, arr)
    if case.geometry is not None and field != "geometry":
        geo = case.geometry.copy()
        geo[k] = 0.0  # a fluid node, so that its codes are read
        case.geometry = geo


def _macro_rho_without_rho(case):
    _set(case, "macro", 11, 8)  # code 8 prescribes rho only
    case.rho = None


def _macro_u_without_u(case):
    _set(case, "macro", 11, 1)  # code 1 prescribes u_x
    case.u = None


BAD = [
    ("MacroBC code above 15", "d3q15", (5, 4, 3), lambda c: _set(c, "macro", 7, 16)),
    ("negative MacroBC code", "d3q15", (5, 4, 3), lambda c: _set(c, "macro", 9, -1)),
    ("MicroBC code above 12", "d3q15", (5, 4, 3), lambda c: _set(c, "micro", 7, 13)),
    ("D2Q9 MicroBC code 3", "d2q9", (8, 6, 1), lambda c: _set(c, "micro", 9, 3)),
    ("non-finite porosity", "d3q15", (5, 4, 3), lambda c: _set(c, "geometry", 5, np.nan)),
    ("rho prescribed, rho absent", "d3q15", (5, 4, 3), _macro_rho_without_rho),
    ("u prescribed, u absent", "d2q9", (8, 6, 1), _macro_u_without_u),
]


@pytest.mark.parametrize("name,lat,length,mutate", BAD, ids=[b[0] for b in BAD])
def test_init_rejects_what_validate_rejects(lbmc, name, lat, length, mutate):
    case = make_case(lat, length, solids=0.1, macro="random", micro="zh", seed=4)
    mutate(case)
    expect = _validate(lbmc, case)
    assert expect[0] == lbmc.ERR_INVALID_ARG, expect
    assert _init_error(lbmc, case) == expect


def test_init_names_the_first_bad_node_across_threads(lbmc):
    """2^20 nodes, so the scan runs on several host threads: three bad nodes
    in different threads' ranges, and the report names the lowest."""
    case = make_case("d2q9", (1024, 1024, 1), solids=0.05, micro="zh", seed=6)
    for k in (900_000, 300_001, 300_000 + 1024 * 512):
        _set(case, "micro", k, 3)
    st, msg = _validate(lbmc, case)
    assert st == lbmc.ERR_INVALID_ARG and "node 300001" in msg, msg
    assert _init_error(lbmc, case) == (st, msg)
    # the engine is usable after the rejection
    good = make_case("d2q9", (64, 32, 1), solids=0.1, micro="zh", seed=6)
    with lbmc.Engine.from_case(good) as eng:
        eng.iterate(5, lbmc.STORE_MACROS | lbmc.SYNC)
        assert np.isfinite(eng.rho()).all()
