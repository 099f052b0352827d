"""The benchmark's own workload against the reference's own step.

The headline measurement runs the porous-medium D3Q15 MRT problem
(overlapping spheres of radius 6 up to solid fraction 0.30, Zou-He pressure
faces at rho = 1.001 / 0.999 on x = 0 and x = Lx-1 through MacroBC 8 and
MicroBC 1/2, periodic y and z, tau = 0.7 with s_e = s_eps = 1.19,
s_q = s_m = 1.2, s_nu = 1/tau and zero rates on rho and j) with FP32 storage
in the tiled AA layout.  Here the same generator builds a 64^3 crop
(Lx = 64, so the tiled layout runs) and the engine, through the C ABI, is
held to the host-compiled reference (patched build: the D3Q15 M_inv, -7/3
and +z Zou-He fixes; LBM-C/solver.cu:10-136, collision.cu:192-303,
boundary_conditions/d3q15/d3q15_zh_defs.cu:4-32) for 1000 FP32 steps and
100 FP64 steps.

Error measure: err(X) = max|X_gpu - X_ref| / max|X_ref| over all nodes and
components; density over the fluid nodes (solid nodes hold rho = 0 in both).
Bounds: 1e-5 for FP32 storage after 1000 steps, 1e-10 for FP64 storage.
"""
import numpy as np
import pytest

import workloads
from oracle.oracle import Case, Reference, Restatement, reference_available

pytestmark = pytest.mark.gpu

CROP = (64, 64, 64)


def err(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.abs(a - b).max() / np.abs(b).max())


@pytest.fixture(scope="module")
def porous():
    """The crop, and the reference's rho/u after 100 and 1000 steps."""
    w = workloads.porous_spheres(CROP)
    a = w.arrays
    case = Case(lattice="d3q15", length=CROP, tau=w.tau, tau_mrt=w.tau_mrt, collision_type=2,
                macro_bc=True, micro_bc=True, geometry=a["geometry"], macro=a["macro"],
                micro=a["micro"], rho=a["rho"], u=a["u"])
    ref = Reference(case, "patched") if reference_available("d3q15", "patched") else Restatement(case)
    out = {}
    done = 0
    for steps in (100, 1000):
        ref.run(steps - done)
        done = steps
        rho, u = ref.macros()
        out[steps] = (ref.f() if steps == 100 else None, rho, u)
    return w, case, out


def _run(lbmc, w, steps, storage, streaming):
    eng = workloads.engine_for(lbmc, w, storage, streaming=streaming)
    with eng:
        eng.iterate(steps, lbmc.STORE_MACROS | lbmc.SYNC)
        return eng.f() if steps == 100 else None, eng.rho(), eng.u()


@pytest.mark.parametrize("streaming", ["aa", "shift"])
def test_porous_crop_fp32_1000_steps(lbmc, porous, streaming):
    w, case, ref = porous
    _, rho_ref, u_ref = ref[1000]
    _, rho, u = _run(lbmc, w, 1000, "f32", lbmc.STREAM_AA if streaming == "aa" else lbmc.STREAM_SHIFT)
    fluid = case.geometry < 1
    eu, er = err(u, u_ref), err(rho[fluid], rho_ref[fluid])
    print(f"porous 64^3 FP32 {streaming}, 1000 steps: err(u) = {eu:.3e}, err(rho) = {er:.3e}, "
          f"max|u| = {np.abs(u_ref).max():.3e}")
    assert eu <= 1e-5
    assert er <= 1e-5
    assert np.array_equal(rho[~fluid], rho_ref[~fluid])


def test_porous_crop_fp64_100_steps(lbmc, porous):
    w, case, ref = porous
    f_ref, rho_ref, u_ref = ref[100]
    f, rho, u = _run(lbmc, w, 100, "f64", lbmc.STREAM_AA)
    assert err(f, f_ref) <= 1e-10
    assert err(u, u_ref) <= 1e-10
    fluid = case.geometry < 1
    assert err(rho[fluid], rho_ref[fluid]) <= 1e-10

