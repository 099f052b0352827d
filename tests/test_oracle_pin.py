"""Pins the CPU restatement oracle to the reference.

1. Against tests/golden/*.npz, produced by the reference's own step
   (host-compiled from the reference sources, tests/golden/make_golden.py):
   the restatement must reproduce every fixture bit for bit.
2. Against the host-compiled reference itself (oracle/_ref) on more seeded
   cases, when those libraries are present (they are built here from the
   reference sources and travel with the tree).
3. Lattice invariants of the tables.
"""
import glob
import json
import os

import numpy as np
import pytest

from cases import make_case
from oracle.oracle import (COMPAT_AS_IS, COMPAT_MRTPOR_INPLACE, Case, Reference, Restatement,
                           reference_available)

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))


def load_golden(path):
    z = np.load(path)
    meta = json.loads(str(z["meta"]))
    arrays = {k[3:]: z[k] for k in z.files if k.startswith("in_")}
    case = Case(lattice=meta["lattice"], length=tuple(meta["length"]), tau=meta["tau"],
                tau_mrt=tuple(meta["tau_mrt"]), c_smag=meta["c_smag"],
                collision_type=meta["collision_type"], forcing=meta["forcing"],
                macro_bc=meta["macro_bc"], micro_bc=meta["micro_bc"], compat=meta["compat"],
                geometry=arrays.get("geometry"), force=arrays.get("force"),
                macro=arrays.get("macro"), micro=arrays.get("micro"), u=arrays.get("u"),
                rho=arrays.get("rho"), f0=arrays.get("f0"))
    return meta, case, z["out_f"], z["out_rho"], z["out_u"]


def test_golden_fixtures_present():
    assert len(GOLDEN) >= 20


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_restatement_matches_golden_bitwise(path):
    meta, case, f, rho, u = load_golden(path)
    r = Restatement(case)
    r.run(meta["nsteps"], store_last=True)
    rr, ur = r.macros()
    np.testing.assert_array_equal(r.f(), f)
    np.testing.assert_array_equal(rr, rho)
    np.testing.assert_array_equal(ur, u)


LIVE = [(lat, ct, forcing, bc, smag)
        for lat in ("d2q9", "d3q15") for ct in range(4) for forcing in (False, True)
        for bc in (None, "random", "zh") for smag in (0.0, 0.1) if not (smag and ct >= 2)]


@pytest.mark.parametrize("lat,ct,forcing,bc,smag", LIVE)
def test_restatement_matches_reference_live(lat, ct, forcing, bc, smag):
    variant = "patched" if smag else "asis"
    if not reference_available(lat, variant):
        pytest.skip("oracle/_ref not built (needs the reference sources)")
    length = (13, 6, 1) if lat == "d2q9" else (6, 5, 4)
    case = make_case(lat, length, ct, forcing, solids=0.12, partial=0.2 if ct % 2 else 0.0,
                     macro="random" if bc == "random" else None,
                     micro="zh" if bc == "zh" else None, c_smag=smag, seed=101 + ct)
    case.compat = COMPAT_AS_IS if variant == "asis" else COMPAT_MRTPOR_INPLACE
    r = Restatement(case)
    r.run(9)
    ref = Reference(case, variant, nthreads=2)
    ref.run(9)
    np.testing.assert_array_equal(r.f(), ref.f())
    (a, b), (c, d) = r.macros(), ref.macros()
    np.testing.assert_array_equal(a, c)
    np.testing.assert_array_equal(b, d)


@pytest.mark.parametrize("lat,ct,forcing,bc", [
    (lat, ct, forcing, bc) for lat in ("d2q9", "d3q15") for ct in (2, 3)
    for forcing in (False, True) for bc in (None, "random", "zh")])
def test_restatement_matches_reference_live_conserved_mrt_rates(lat, ct, forcing, bc):
    """MRT with non-zero rates on rho and j (a TauMRT line that sets them),
    against the patched reference: the D3Q15 as-is reference relaxes nothing
    (its M_inv is zero), so only the patched build exercises these rates."""
    if not reference_available(lat, "patched"):
        pytest.skip("oracle/_ref not built (needs the reference sources)")
    length = (13, 6, 1) if lat == "d2q9" else (6, 5, 4)
    case = make_case(lat, length, ct, forcing, solids=0.12, partial=0.2 if ct == 3 else 0.0,
                     macro="random" if bc == "random" else None,
                     micro="zh" if bc == "zh" else None, seed=301 + ct, mrt_conserved=1.05)
    case.compat = COMPAT_MRTPOR_INPLACE
    r = Restatement(case)
    r.run(9)
    ref = Reference(case, "patched", nthreads=2)
    ref.run(9)
    np.testing.assert_array_equal(r.f(), ref.f())
    (a, b), (c, d) = r.macros(), ref.macros()
    np.testing.assert_array_equal(a, c)
    np.testing.assert_array_equal(b, d)


@pytest.mark.parametrize("lat", ["d2q9", "d3q15"])
def test_lattice_invariants(lat):
    case = make_case(lat, (4, 4, 4))
    e, w, opp, M, Minv = Restatement(case).tables()
    q = case.q
    assert abs(w.sum() - 1) < 1e-15
    assert np.all(opp[opp] == np.arange(q))
    assert np.all(e[:, opp] == -e)
    np.testing.assert_allclose(M @ Minv, np.eye(q), atol=1e-14)
    # rows of M are orthogonal: M^-1 = M^T D^-1
    D = (M * M).sum(1)
    np.testing.assert_allclose(Minv, M.T / D[None, :], atol=1e-15)


def test_reference_d3q15_minv_is_zero_as_is():
    """Defect Q1: the reference's D3Q15 M_inv literals are integer divisions."""
    case = make_case("d3q15", (4, 4, 4), compat=COMPAT_AS_IS)
    *_, Minv = Restatement(case).tables()
    assert np.abs(Minv).sum() == 0.0


def test_shift_map_is_a_bijection():
    """Every (population, step) maps nodes one to one onto slots."""
    L = np.array([7, 5, 3])
    e = np.array([[0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1],
                  [0, 0, 0, 1, -1, 0, 0, 1, 1, -1, -1, 1, 1, -1, -1],
                  [0, 0, 0, 0, 0, 1, -1, 1, 1, 1, 1, -1, -1, -1, -1]])
    c = np.stack(np.meshgrid(*[np.arange(l) for l in L], indexing="ij")).reshape(3, -1)
    for t in (0, 1, 6, 23):
        for i in range(15):
            s = np.mod(c - t * e[:, i:i + 1], L[:, None])
            idx = s[0] + L[0] * (s[1] + L[1] * s[2])
            assert len(np.unique(idx)) == c.shape[1]
