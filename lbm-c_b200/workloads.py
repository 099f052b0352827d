"""Seeded synthetic workloads with the shapes of the benchmark configurations.

No public dataset is involved: each workload is generated from a seed with
the sizes, parameters and value distributions of the configuration it stands
for.  Arrays follow the reference's node order ixd = x + y*Lx + z*Lx*Ly.

* ``poiseuille_channel``  D2Q9 BGK + Guo, 128x64, tau 0.8, g_x 1e-6, walls at
  y = 0 and y = Ly-1, periodic x.
* ``porous_spheres``      D3Q15 MRT, 256^3, overlapping spheres (radius 6,
  uniform centres) up to solid fraction 0.30, Zou-He rho = 1.001 / 0.999 on
  the x faces (MacroBC 8 + MicroBC 1/2), periodic y/z, tau 0.7,
  s_e = s_eps = 1.19, s_q = 1.2, s_nu = 1/tau, s_m = 1.2.
* ``taylor_green``        D3Q15 BGK + Smagorinsky C_s = 0.1, periodic cube,
  Re 1600, u0 0.05.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


@dataclass
class Workload:
    name: str
    lattice: str
    length: tuple
    tau: float
    collision_type: int
    tau_mrt: tuple = ()
    c_smag: float = 0.0
    forcing: bool = False
    macro_bc: bool = False
    micro_bc: bool = False
    init_type: int = 0
    arrays: dict = field(default_factory=dict)  # geometry, force, macro, micro, u, rho, f0
    params: dict = field(default_factory=dict)

    @property
    def dim(self):
        return 2 if self.lattice == "d2q9" else 3

    @property
    def q(self):
        return 9 if self.lattice == "d2q9" else 15

    @property
    def n(self):
        return int(np.prod(self.length[:self.dim]))

    def host_bytes(self):
        return sum(a.nbytes for a in self.arrays.values() if a is not None)


def poiseuille_channel(lx=128, ly=64, tau=0.8, g=1e-6) -> Workload:
    n = lx * ly
    y = np.arange(n) // lx
    geometry = np.zeros(n)
    geometry[(y == 0) | (y == ly - 1)] = 1.0
    force = np.zeros((2, n))
    force[0] = g
    return Workload("poiseuille_d2q9_bgk_guo", "d2q9", (lx, ly, 1), tau, 0, forcing=True,
                    arrays=dict(geometry=geometry, force=force),
                    params=dict(g=g, nu=(tau - 0.5) / 3))


def sphere_pack(L=(256, 256, 256), radius=6, target=0.30, seed=2024, keep_x_faces=True):
    """Boolean solid mask (z, y, x) of overlapping spheres with uniform
    centres, added in batches until the solid fraction reaches target.
    Spheres wrap periodically in y and z; the x = 0 and x = Lx-1 planes stay
    fluid so the pressure faces are well posed."""
    lx, ly, lz = L
    rng = np.random.default_rng(seed)
    solid = np.zeros((lz, ly, lx), bool)
    r = radius
    d = np.arange(-r, r + 1)
    dz, dy, dx = np.meshgrid(d, d, d, indexing="ij")
    ball = (dx * dx + dy * dy + dz * dz) <= r * r
    bz, by, bx = dz[ball], dy[ball], dx[ball]
    # Boolean-model estimate of the sphere count, then top up in batches.
    vol = ball.sum()
    nsph = int(-np.log(1 - target) * lx * ly * lz / vol)
    count = 0
    while True:
        cx = rng.uniform(0, lx, nsph).astype(int)
        cy = rng.uniform(0, ly, nsph).astype(int)
        cz = rng.uniform(0, lz, nsph).astype(int)
        X = cx[:, None] + bx[None]
        Y = (cy[:, None] + by[None]) % ly
        Z = (cz[:, None] + bz[None]) % lz
        ok = (X >= 0) & (X < lx)
        solid[Z[ok], Y[ok], X[ok]] = True
        count += nsph
        if keep_x_faces:
            solid[:, :, 0] = False
            solid[:, :, lx - 1] = False
        frac = solid.mean()
        if frac >= target:
            break
        nsph = max(16, int(nsph * 0.05))
    return solid, count


def porous_spheres(L=(256, 256, 256), tau=0.7, rho_in=1.001, rho_out=0.999, seed=2024,
                   radius=6, target=0.30) -> Workload:
    lx, ly, lz = L
    n = lx * ly * lz
    solid, count = sphere_pack(L, radius, target, seed)
    geometry = solid.reshape(n).astype(np.float64)
    x = np.arange(n) % lx
    macro = np.zeros(n, np.int32)
    micro = np.zeros(n, np.int32)
    rho = np.ones(n)
    inlet, outlet = x == 0, x == lx - 1
    macro[inlet | outlet] = 8  # presc_rho (macro_bc.cu:67-70)
    micro[inlet] = 1           # zh_pressure_x
    micro[outlet] = 2          # zh_pressure_X
    rho[inlet] = rho_in
    rho[outlet] = rho_out
    s_nu = 1.0 / tau
    tau_mrt = (0.0, 1.19, 1.19, 0.0, 1.2, 0.0, 1.2, 0.0, 1.2,
               s_nu, s_nu, s_nu, s_nu, s_nu, 1.2)
    return Workload("porous_spheres_d3q15_mrt", "d3q15", tuple(L), tau, 2, tau_mrt=tau_mrt,
                    macro_bc=True, micro_bc=True,
                    arrays=dict(geometry=geometry, macro=macro, micro=micro, rho=rho,
                                u=np.zeros((3, n))),
                    params=dict(solid_fraction=float(solid.mean()), spheres=count,
                                rho_in=rho_in, rho_out=rho_out))


def taylor_green(L=256, u0=0.05, re=1600.0, c_smag=0.1) -> Workload:
    """Periodic cube with u = u0 sin x cos y cos z, v = -u0 cos x sin y cos z,
    w = 0 and p = p0 + rho0 u0^2/16 (cos 2x + cos 2y)(cos 2z + 2), mapped to
    rho = 1 + 3 (p - p0); populations start at f_eq(rho, u)."""
    n = L ** 3
    k = 2 * np.pi / L
    ell = L / (2 * np.pi)
    nu = u0 * ell / re
    tau = 3 * nu + 0.5
    c = (np.arange(L) + 0.5) * k
    z, y, x = np.meshgrid(c, c, c, indexing="ij")
    u = np.empty((3, n))
    u[0] = (u0 * np.sin(x) * np.cos(y) * np.cos(z)).reshape(n)
    u[1] = (-u0 * np.cos(x) * np.sin(y) * np.cos(z)).reshape(n)
    u[2] = 0
    p = (u0 * u0 / 16) * (np.cos(2 * x) + np.cos(2 * y)) * (np.cos(2 * z) + 2)
    rho = 1 + 3 * p.reshape(n)
    return Workload("taylor_green_d3q15_bgk_smag", "d3q15", (L, L, L), tau, 0, c_smag=c_smag,
                    init_type=1, arrays=dict(u=u, rho=rho),
                    params=dict(nu=nu, u0=u0, re=re, ell=ell))


def forced_box(L=128, tau=0.5025, amp=1.6e-5, c_smag=0.1, seed=1) -> Workload:
    """Periodic D3Q15 BGK box driven by a static solenoidal Guo force of
    random Fourier modes |k| <= 2 (the closure study's coarse grid);
    Smagorinsky C_s = c_smag where a learned closure's inputs leave its
    range."""
    import closure
    force = closure.fourier_force(L, amp, 2, seed)
    return Workload("forced_box_d3q15_bgk", "d3q15", (L, L, L), tau, 0, c_smag=c_smag, forcing=True,
                    arrays=dict(force=force), params=dict(amp=amp, seed=seed))


def engine_for(lbmc, w: Workload, storage="f32", **kw):
    """lbmc.Engine for a workload (lbmc is the binding module)."""
    a = w.arrays
    cfg = lbmc.make_config(w.lattice, w.length, tau=w.tau, tau_mrt=w.tau_mrt, c_smag=w.c_smag,
                           collision_type=w.collision_type, forcing=w.forcing,
                           macro_bc=w.macro_bc, micro_bc=w.micro_bc, init_type=w.init_type,
                           storage=lbmc.STORAGE_IDS.get(storage, storage), **kw)
    dom, keep = lbmc.make_domain(w.n, w.dim, w.q, a.get("geometry"), a.get("force"),
                                 a.get("macro"), a.get("micro"), a.get("u"), a.get("rho"),
                                 a.get("f0"))
    eng = lbmc.Engine(cfg, dom)
    del keep
    return eng


def imb_weight(eps, tau):
    """Noble-Torczynski solid weight from area coverage:
    B = eps (tau - 1/2) / ((1 - eps) + (tau - 1/2)); eps = 1 gives B = 1."""
    return eps * (tau - 0.5) / ((1.0 - eps) + (tau - 0.5))


def circle_domain(lx, ly, target, rng, rmin=3.0, rmax=12.0, tau=1.0):
    """Porosity field (ly, lx) of random circles (radius U[rmin, rmax], uniform
    periodic centres) added until the covered area reaches `target`.  Cell
    coverage eps = clamp(r - |x_cell - c| + 1/2, 0, 1) (signed-distance area
    estimate), union by maximum; B from imb_weight."""
    eps = np.zeros((ly, lx))
    while eps.mean() < target:
        r = rng.uniform(rmin, rmax)
        cx, cy = rng.uniform(0, lx), rng.uniform(0, ly)
        R = int(np.ceil(r + 1))
        xs = np.arange(int(np.floor(cx)) - R, int(np.floor(cx)) + R + 1)
        ys = np.arange(int(np.floor(cy)) - R, int(np.floor(cy)) + R + 1)
        dx = (xs + 0.5 - cx)[None, :]
        dy = (ys + 0.5 - cy)[:, None]
        cov = np.clip(r - np.sqrt(dx * dx + dy * dy) + 0.5, 0.0, 1.0)
        ix, iy = np.mod(xs, lx), np.mod(ys, ly)
        sub = eps[np.ix_(iy, ix)]
        eps[np.ix_(iy, ix)] = np.maximum(sub, cov)
    return imb_weight(eps, tau)


def batch_sweep(n=4096, lmin=32, lmax=512, seed=5, tau=1.0, square=False):
    """Batched-sweep domains: sides log-uniform in [lmin, lmax] (independent
    per axis unless square), solid fraction U[0.2, 0.5] of circles radius
    3-12 with IMB edges."""
    rng = np.random.default_rng(seed)
    geoms = []
    for _ in range(n):
        lx = int(round(np.exp(rng.uniform(np.log(lmin), np.log(lmax)))))
        ly = lx if square else int(round(np.exp(rng.uniform(np.log(lmin), np.log(lmax)))))
        geoms.append(circle_domain(lx, ly, rng.uniform(0.2, 0.5), rng, tau=tau))
    return geoms
