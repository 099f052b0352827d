"""Seeded synthetic time-step problems shared by the CPU and GPU tests.

Every case is a ``oracle.oracle.Case``: arrays in the reference's ixd order
(x fastest), populations in natural layout.  Nothing here reads the
reference tree; fixtures made from the reference live in tests/golden/.
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from oracle.oracle import Case, LATTICES  # noqa: E402

E = {
    "d2q9": np.array([[0, 1, 0, -1, 0, 1, -1, -1, 1],
                      [0, 0, 1, 0, -1, 1, 1, -1, -1]]),
    "d3q15": np.array([[0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1],
                       [0, 0, 0, 1, -1, 0, 0, 1, 1, -1, -1, 1, 1, -1, -1],
                       [0, 0, 0, 0, 0, 1, -1, 1, 1, 1, 1, -1, -1, -1, -1]]),
}
W = {
    "d2q9": np.array([4 / 9] + [1 / 9] * 4 + [1 / 36] * 4),
    "d3q15": np.array([2 / 9] + [1 / 9] * 6 + [1 / 72] * 8),
}
# The porous benchmark's MRT rates: s_e = s_eps = 1.19, s_q = 1.2, s_nu = 1/tau,
# s_m = 1.2, conserved moments 0.  With conserved = c the rates on rho and j
# are c instead, as a TauMRT input line sets them (e.g. "TauMRT 1.0 1.19 1.19
# 1.0 1.2 1.0 1.2 1.25 1.25"); the reference relaxes every moment with its
# rate (LBM-C/collision.cu:192-303), so non-zero conserved rates act wherever
# m_k differs from its equilibrium (with Guo forcing, j - rho u = -F/2).
def mrt_rates(lattice: str, tau: float, conserved: float = 0.0):
    c = conserved
    if lattice == "d2q9":
        # rho, e, eps, jx, qx, jy, qy, pxx, pxy
        return (c, 1.19, 1.19, c, 1.2, c, 1.2, 1 / tau, 1 / tau)
    return (c, 1.19, 1.19, c, 1.2, c, 1.2, c, 1.2,
            1 / tau, 1 / tau, 1 / tau, 1 / tau, 1 / tau, 1.2)


def equilibrium(lattice: str, rho, u):
    e, w = E[lattice], W[lattice]
    eu = 3.0 * np.einsum("dq,dn->qn", e, u)
    usq = 1.5 * (u * u).sum(0)
    return rho[None] * w[:, None] * (1.0 + eu + 0.5 * eu * eu - usq[None])


def make_case(lattice: str = "d2q9", length=(16, 12, 1), collision_type: int = 0,
              forcing: bool = False, solids: float = 0.0, partial: float = 0.0,
              macro: str | None = None, micro: str | None = None, c_smag: float = 0.0,
              tau: float = 0.8, seed: int = 0, uniform_force: bool = False,
              u_amp: float = 0.02, compat: int = 0, mrt_conserved: float = 0.0) -> Case:
    """A random near-equilibrium state with the requested options.

    macro: None | "random" (codes 1..15 at ~6% of nodes) | "zh" (rho on faces)
    micro: None | "zh" (Zou-He pressure faces) | "sf" (stress-free faces)
    mrt_conserved: MRT rate on rho and j (0 = the benchmark's rates)
    """
    _, dim, q = LATTICES[lattice]
    length = tuple(length[:dim]) + (1,) * (3 - dim)
    n = int(np.prod(length[:dim]))
    rng = np.random.default_rng(seed)
    rho0 = 1.0 + 0.01 * rng.standard_normal(n)
    u0 = u_amp * rng.standard_normal((dim, n))
    f0 = equilibrium(lattice, rho0, u0) + 1e-3 * W[lattice][:, None] * rng.standard_normal((q, n))
    case = Case(lattice=lattice, length=length, tau=tau, collision_type=collision_type,
                forcing=forcing, c_smag=c_smag, compat=compat, f0=f0)
    if collision_type >= 2:
        case.tau_mrt = mrt_rates(lattice, tau, mrt_conserved)
    geometry = np.zeros(n)
    if solids > 0:
        geometry[rng.random(n) < solids] = 1.0
    if partial > 0:
        mask = (rng.random(n) < partial) & (geometry < 1)
        geometry[mask] = rng.uniform(0.05, 0.95, mask.sum())
    case.geometry = geometry
    if forcing:
        if uniform_force:
            case.force = np.tile(np.array([1e-4, -5e-5, 2e-5][:dim])[:, None], (1, n))
        else:
            case.force = 1e-4 * rng.standard_normal((dim, n))
    coords = np.stack(np.unravel_index(np.arange(n), length[:dim][::-1])[::-1])  # (dim, n): x, y[, z]
    macro_codes = np.zeros(n, np.int32)
    micro_codes = np.zeros(n, np.int32)
    if macro == "random":
        mask = rng.random(n) < 0.06
        codes = rng.integers(1, 16, n)
        macro_codes[mask] = codes[mask]
    if micro in ("zh", "sf"):
        nfaces = 2 if lattice == "d2q9" and micro == "zh" else 2 * dim
        for face in range(nfaces):
            axis, hi = face // 2, face % 2
            sel = coords[axis] == (length[axis] - 1 if hi else 0)
            # lower-numbered faces win at edges and corners
            sel &= micro_codes == 0
            if micro == "zh":
                code = face + 1
            else:
                code = (5 if lattice == "d2q9" else 7) + face
            micro_codes[sel] = code
            if micro == "zh":
                macro_codes[sel] = 8  # presc_rho feeds the Zou-He density
        geometry[micro_codes > 0] = 0.0
    if macro is not None or micro == "zh":
        case.macro_bc = True
        case.macro = macro_codes
        case.rho = 1.0 + 0.002 * rng.standard_normal(n)
        case.u = 0.01 * rng.standard_normal((dim, n))
    if micro is not None:
        case.micro_bc = True
        case.micro = micro_codes
    return case


def poiseuille_channel() -> Case:
    """D2Q9 BGK+Guo Poiseuille channel 128x64, tau 0.8, g_x = 1e-6, walls at
    y = 0 and y = 63 (B = 1), periodic in x, f = w_i (Init 0)."""
    lx, ly = 128, 64
    n = lx * ly
    geometry = np.zeros(n)
    y = np.arange(n) // lx
    geometry[(y == 0) | (y == ly - 1)] = 1.0
    force = np.zeros((2, n))
    force[0] = 1e-6
    return Case(lattice="d2q9", length=(lx, ly, 1), tau=0.8, collision_type=0,
                forcing=True, geometry=geometry, force=force)


def poiseuille_startup(y, t, g=1e-6, nu=0.1, h=62.0, y0=0.5, nterms=200):
    """Transient body-force channel flow from rest between walls at y0 and
    y0 + h: u = g/(2nu) eta (h - eta) - sum_{n odd} 4 g h^2/(nu pi^3 n^3)
    sin(n pi eta/h) exp(-n^2 pi^2 nu t / h^2)."""
    eta = np.asarray(y, float) - y0
    u = g / (2 * nu) * eta * (h - eta)
    for k in range(1, 2 * nterms, 2):
        u -= 4 * g * h * h / (nu * np.pi ** 3 * k ** 3) * np.sin(k * np.pi * eta / h) * \
            np.exp(-k * k * np.pi * np.pi * nu * t / (h * h))
    return np.where((eta > 0) & (eta < h), u, 0.0)
