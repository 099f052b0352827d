"""Accuracy studies of the reduced-precision storages against an FP64 run
of the same engine at the same size (the FP64 storage computes and stores
in FP64 throughout).

- porous_accuracy: D3Q15 MRT flow through the random sphere pack with Zou-He
  pressure faces (the 256^3 benchmark case), N steps per storage; velocity
  error against FP64 and the Darcy permeability
      k = nu <u_x> (Lx - 1) / (c_s^2 (rho_in - rho_out)),
  <u_x> the superficial (whole-volume) mean velocity over the interior
  planes, c_s^2 = 1/3, rho0 = 1.
- tgv_accuracy: the Taylor-Green vortex (D3Q15 BGK + Smagorinsky, periodic
  L^3, Re 1600, u0 0.05) for a number of convective times T_c = L/(2 pi u0);
  kinetic energy from the engine's fused FP64 sum every 0.1 T_c, enstrophy
  (1/2 <|curl u|^2>, central differences, volume mean) every T_c; errors of
  both decay curves against FP64.
Rates are the lbmc_iterate wall clock of the run's steps (synchronised), not
the bench's event-timed kernel rate.
"""
from __future__ import annotations

import time

import numpy as np

import workloads


def _timed_iterate(lbmc, eng, steps, flags):
    t = time.perf_counter()
    eng.iterate(steps, flags | lbmc.SYNC)
    return time.perf_counter() - t


def porous_accuracy(lbmc, L=256, steps=5000, storages=("f64", "f32", "f16", "f16sr", "bf16"),
                    streaming=None, log=print):
    w = workloads.porous_spheres((L, L, L))
    streaming = lbmc.STREAM_AA if streaming is None else streaming
    nu = (w.tau - 0.5) / 3
    p = w.params
    out, ref = {"nodes": w.n, "steps": steps, "solid_fraction": p["solid_fraction"]}, None
    for st in storages:
        eng = workloads.engine_for(lbmc, w, st, streaming=streaming)
        secs = _timed_iterate(lbmc, eng, steps, lbmc.STORE_MACROS | lbmc.REDUCE_DIAG)
        u, rho = eng.u(), eng.rho()
        eng.close()
        ux = u[0].reshape(L, L, L)[:, :, 1:L - 1]
        k = nu * ux.mean() * (L - 1) / ((p["rho_in"] - p["rho_out"]) / 3)
        r = {"glups_wall": w.n * steps / secs / 1e9, "permeability": float(k),
             "u_mean": float(ux.mean())}
        if ref is None:
            ref = (u, rho, k)
        else:
            u0, rho0, k0 = ref
            r["u_rel_max"] = float(np.abs(u - u0).max() / np.abs(u0).max())
            r["u_rel_l2"] = float(np.linalg.norm(u - u0) / np.linalg.norm(u0))
            r["rho_rel_max"] = float(np.abs(rho - rho0).max() / np.abs(rho0 - 1).max())
            r["permeability_rel"] = float(abs(k - k0) / abs(k0))
        out[st] = r
        log(f"porous {L}^3 {st}: {r}")
    return out


def _enstrophy(torch, u, L):
    """1/2 <|curl u|^2> by central differences (periodic, dx = 1); u is
    (3, L^3) in node order x + L (y + L z)."""
    U = torch.as_tensor(u, dtype=torch.float64, device="cuda").reshape(3, L, L, L)  # (c, z, y, x)

    def d(a, axis):  # axis 0 = x, 1 = y, 2 = z
        dim = 2 - axis
        return 0.5 * (torch.roll(a, -1, dims=dim) - torch.roll(a, 1, dims=dim))
    wx = d(U[2], 1) - d(U[1], 2)
    wy = d(U[0], 2) - d(U[2], 0)
    wz = d(U[1], 0) - d(U[0], 1)
    return float(0.5 * (wx * wx + wy * wy + wz * wz).mean())


def tgv_accuracy(lbmc, torch, L=512, conv_times=20, storages=("f64", "f32", "f16", "f16sr", "bf16"),
                 streaming=None, log=print):
    w = workloads.taylor_green(L)
    streaming = lbmc.STREAM_AA if streaming is None else streaming
    u0 = w.params["u0"]
    tc = L / (2 * np.pi * u0)
    ke_points = [int(round(0.1 * j * tc)) for j in range(1, 10 * conv_times + 1)]
    en_points = set(int(round(j * tc)) for j in range(1, conv_times + 1))
    a = w.arrays
    ke_init = float(0.5 * (a["rho"] * (a["u"] ** 2).sum(0)).sum())
    out = {"L": L, "tau": w.tau, "nu": w.params["nu"], "T_c_steps": tc, "steps": ke_points[-1],
           "ke_initial": ke_init}
    ref = None
    for st in storages:
        eng = workloads.engine_for(lbmc, w, st, streaming=streaming)
        done, secs = 0, 0.0
        ke, en = [], []
        for s in ke_points:
            store = s in en_points
            secs += _timed_iterate(lbmc, eng, s - done,
                                   lbmc.REDUCE_DIAG | (lbmc.STORE_MACROS if store else 0))
            done = s
            ke.append(eng.diag().kinetic_energy)
            if store:
                en.append(_enstrophy(torch, eng.u(), L))
        eng.close()
        ke, en = np.array(ke), np.array(en)
        r = {"glups_wall": w.n * done / secs / 1e9, "ke_final_over_initial": float(ke[-1] / ke_init),
             "enstrophy_peak": float(en.max()),
             "enstrophy_peak_tc": float((1 + int(en.argmax()))),
             "ke": ke.tolist()[::10], "enstrophy": en.tolist()}
        if ref is None:
            ref = (ke, en)
        else:
            k0, e0 = ref
            r["ke_err_max"] = float(np.abs(ke - k0).max() / ke_init)
            r["enstrophy_err_max"] = float(np.abs(en - e0).max() / e0.max())
            r["dissipation_err_max"] = float(np.abs(np.diff(ke) - np.diff(k0)).max() / np.abs(np.diff(k0)).max())
        out[st] = r
        log(f"tgv {L}^3 {st}: " + str({k: v for k, v in r.items() if k not in ('ke', 'enstrophy')}))
    return out
