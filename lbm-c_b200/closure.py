"""Learned subgrid closure: training data from this solver, training, and the
coarse-grid comparison against Smagorinsky and the filtered fine solve.

Pipeline (all on one GPU; torch only prepares data, the solver and the
network run in liblbmc):

1. Fine solve: D3Q15 BGK forced isotropic turbulence, periodic box, Guo force
   from random solenoidal Fourier modes |k| <= kmax (amplitudes N(0, amp),
   seeded phases), rest start; snapshots of rho and u.  At tau = 0.51 on 256^3
   an amplitude of 1e-5 drives u_rms past BGK's stability limit (non-finite
   state at step 12000); 4e-6 settles at u_rms ~ 0.04-0.055 and is the
   default.
2. Box filter by `factor` to the coarse grid: u_bar, rho_bar and the subgrid
   stress tau_ij = bar(u_i u_j) - u_bar_i u_bar_j; filtered strain S_bar by
   central differences on the coarse grid.
3. Target: the least-squares eddy viscosity nu* = max(0, -dev(tau):S_bar /
   (2 S_bar:S_bar)) per coarse cell; inputs: six invariants of S_bar and
   rho_bar (lbmc_mlp_features, the same device function the step uses).
4. Train the 6-32-32-1 network (lbmc_mlp_train), normalisation from the data,
   training range = central 99.8% of each normalised input.
5. Coarse runs from a filtered snapshot of an independent fine solve (other
   seed): no model, Smagorinsky (C_s = 0.1) and the learned closure, and
   Smagorinsky on the finer grid whose wall clock matches the learned run's;
   errors against the filtered fine solution.

Units: acoustic scaling (dx, dt both x factor) keeps velocities; the coarse
viscosity is nu_fine / factor and the coarse force factor x filtered force.
"""
from __future__ import annotations

import time

import numpy as np


def fourier_force(L, amp=4e-6, kmax=2, seed=0):
    """Static solenoidal force field (3, L^3) from random Fourier modes."""
    rng = np.random.default_rng(seed)
    c = np.arange(L) * (2 * np.pi / L)
    z, y, x = np.meshgrid(c, c, c, indexing="ij")
    F = np.zeros((3, L, L, L))
    for kx in range(-kmax, kmax + 1):
        for ky in range(-kmax, kmax + 1):
            for kz in range(0, kmax + 1):
                k = np.array([kx, ky, kz], float)
                kk = np.sqrt((k * k).sum())
                if kk == 0 or kk > kmax or (kz == 0 and (ky < 0 or (ky == 0 and kx < 0))):
                    continue
                a = rng.normal(0, amp, 3)
                a -= k * (a @ k) / (kk * kk)  # solenoidal
                ph = rng.uniform(0, 2 * np.pi)
                arg = kx * x + ky * y + kz * z + ph
                F += a[:, None, None, None] * np.cos(arg)[None]
    return F.reshape(3, -1)


def fine_solve(lbmc, L, tau, steps, snap_steps, force, storage="f32"):
    """Runs the fine D3Q15 BGK solve; returns {step: (rho, u)} (host float64)."""
    n = L ** 3
    cfg = lbmc.make_config("d3q15", (L, L, L), tau=tau, collision_type=lbmc.BGK, forcing=True,
                           storage=storage)
    dom, keep = lbmc.make_domain(n, 3, 15, None, force)
    out = {}
    with lbmc.Engine(cfg, dom) as eng:
        done = 0
        for s in sorted(snap_steps):
            eng.iterate(s - done, lbmc.STORE_MACROS | lbmc.REDUCE_DIAG | lbmc.SYNC)
            done = s
            out[s] = (eng.rho(), eng.u())
        if done < steps:
            eng.iterate(steps - done, lbmc.SYNC)
    del keep
    return out


def filtered(torch, rho, u, L, factor, dev):
    """Box-filtered rho, u (coarse, torch) and the subgrid stress tau_ij (6, ...)."""
    Lc = L // factor
    r = torch.as_tensor(rho, device=dev).reshape(L, L, L)
    U = torch.as_tensor(u, device=dev).reshape(3, L, L, L)

    def box(a):
        return a.reshape(Lc, factor, Lc, factor, Lc, factor).mean(dim=(1, 3, 5))
    rb = box(r)
    ub = torch.stack([box(U[d]) for d in range(3)])
    pairs = [(0, 0), (1, 1), (2, 2), (0, 1), (1, 2), (0, 2)]
    tau = torch.stack([box(U[a] * U[b]) - ub[a] * ub[b] for a, b in pairs])
    return rb, ub, tau


def strain_rate(torch, ub):
    """S_ij = (d_i u_j + d_j u_i)/2 by central differences (periodic, dx = 1);
    arrays are indexed (z, y, x).  Order xx, yy, zz, xy, yz, xz."""
    def d(a, axis):  # axis 0 = x, 1 = y, 2 = z
        dim = 2 - axis
        return 0.5 * (torch.roll(a, -1, dims=dim) - torch.roll(a, 1, dims=dim))
    g = [[d(ub[j], i) for j in range(3)] for i in range(3)]  # g[i][j] = d_i u_j
    pairs = [(0, 0), (1, 1), (2, 2), (0, 1), (1, 2), (0, 2)]
    return torch.stack([0.5 * (g[a][b] + g[b][a]) for a, b in pairs])


def optimal_nu(torch, tau, S):
    """Least-squares nu* with dev(tau) ~ -2 nu S (contractions count the
    off-diagonal pairs twice)."""
    tr = (tau[0] + tau[1] + tau[2]) / 3
    dev = tau.clone()
    dev[:3] -= tr
    w = torch.tensor([1, 1, 1, 2, 2, 2], dtype=tau.dtype, device=tau.device).reshape(6, 1, 1, 1)
    num = -(w * dev * S).sum(0)
    den = 2 * (w * S * S).sum(0) + 1e-30
    return torch.clamp(num / den, min=0.0)


def dataset(lbmc, torch, snaps, L, factor, dev):
    """(features (n, 6), nu* (n)) from fine snapshots."""
    X, y = [], []
    for rho, u in snaps:
        rb, ub, tau = filtered(torch, rho, u, L, factor, dev)
        S = strain_rate(torch, ub)
        nu = optimal_nu(torch, tau, S)
        S6 = S.reshape(6, -1).T.contiguous().float().cpu().numpy()
        X.append(lbmc.mlp_features(S6, rb.reshape(-1).float().cpu().numpy()))
        y.append(nu.reshape(-1).float().cpu().numpy())
    return np.concatenate(X), np.concatenate(y)


def train_closure(lbmc, X, y, epochs=8, batch=4096, lr=2e-3, seed=0):
    """Trains the network on (features, nu*); returns (Mlp, loss history)."""
    mean, std = X.mean(0), X.std(0) + 1e-12
    xn = (X - mean) / std
    lo, hi = np.percentile(xn, 0.1, axis=0), np.percentile(xn, 99.9, axis=0)
    scale = float(np.std(y) + 1e-30)
    m = lbmc.Mlp(seed=seed)
    m.set_normalization(mean, std, lo, hi, target_scale=scale)
    hist = m.train(X, y, epochs=epochs, batch=batch, lr=lr)
    return m, hist


def a_priori(lbmc, torch, model, rho, u, L, factor, dev, c_smag=0.1):
    """Held-out comparison of the modelled eddy viscosity with nu* on one
    filtered snapshot: relative L2 error of nu_t and of the subgrid
    dissipation 2 nu_t S:S, and the correlation with nu*, for the learned
    network as the step evaluates it (Smagorinsky where its inputs leave the
    training range) and for Smagorinsky alone (nu = C_s^2 |S|,
    |S| = sqrt(2 S:S))."""
    rb, ub, tau = filtered(torch, rho, u, L, factor, dev)
    S = strain_rate(torch, ub)
    nu_star = optimal_nu(torch, tau, S).reshape(-1).double().cpu().numpy()
    S6 = S.reshape(6, -1).T.contiguous().double().cpu().numpy()
    ss = (S6[:, :3] ** 2).sum(1) + 2 * (S6[:, 3:] ** 2).sum(1)
    nu_smag = c_smag ** 2 * np.sqrt(2 * ss)
    X = lbmc.mlp_features(S6.astype(np.float32), rb.reshape(-1).float().cpu().numpy())
    mean, std, lo, hi = (np.asarray(a, np.float64) for a in model._norm)
    xn = (X - mean) / std
    inside = np.all((xn >= lo) & (xn <= hi), 1)
    nu_learn = np.where(inside, np.maximum(0.0, model.predict_step(X).astype(np.float64)), nu_smag)

    def score(nu):
        return {"nu_rel_l2": float(np.linalg.norm(nu - nu_star) / np.linalg.norm(nu_star)),
                "dissipation_rel_l2": float(np.linalg.norm((nu - nu_star) * ss)
                                            / np.linalg.norm(nu_star * ss)),
                "corr": float(np.corrcoef(nu, nu_star)[0, 1])}
    return {"learned": score(nu_learn), "smagorinsky": score(nu_smag),
            "inside_range": float(inside.mean())}


def fourier_resample(torch, a, N):
    """Band-limited resampling of periodic fields a (C, n, n, n) (torch) to
    N^3: Fourier coefficients |k_i| < min(n, N) / 2 kept, the rest zero."""
    n = a.shape[-1]
    A = torch.fft.rfftn(a, dim=(1, 2, 3), norm="forward")
    m = min(n, N) // 2  # modes -m+1 .. m-1 on the full axes, 0 .. m-1 on the half axis
    src = torch.tensor(list(range(0, m)) + list(range(n - m + 1, n)), device=a.device)
    dst = torch.tensor(list(range(0, m)) + list(range(N - m + 1, N)), device=a.device)
    sub = A[:, src][:, :, src][:, :, :, :m]
    out = torch.zeros((a.shape[0], N, N, N // 2 + 1), dtype=A.dtype, device=A.device)
    tmp = torch.zeros((a.shape[0], N, N, m), dtype=A.dtype, device=A.device)
    tmp[:, dst[:, None], dst[None, :], :] = sub
    out[:, :, :, :m] = tmp
    return torch.fft.irfftn(out, s=(N, N, N), dim=(1, 2, 3), norm="forward")


def coarse_solve(lbmc, rb, ub, Fc, tau_c, checkpoints, model=None, c_smag=0.0, passes=2,
                 storage="f32"):
    """Coarse run from (rho_bar, u_bar) with model None, 'smag' or an Mlp;
    returns ({step: u}, wall-clock seconds of all steps) or (None, nan) if
    the state became non-finite."""
    Lc = rb.shape[0]
    n = Lc ** 3
    cfg = lbmc.make_config("d3q15", (Lc, Lc, Lc), tau=tau_c, collision_type=lbmc.BGK,
                           forcing=True, init_type=lbmc.INIT_EQUILIBRIUM,
                           c_smag=c_smag, storage=storage)
    dom, keep = lbmc.make_domain(n, 3, 15, None, Fc, u=ub.reshape(3, -1), rho=rb.reshape(-1))
    out, wall = {}, 0.0
    with lbmc.Engine(cfg, dom) as eng:
        if model is not None and model != "smag":
            model.attach(eng, iterations=passes)
        done = 0
        for s in sorted(checkpoints):
            t = time.perf_counter()
            eng.iterate(s - done, lbmc.STORE_MACROS | lbmc.SYNC)
            wall += time.perf_counter() - t
            done = s
            out[s] = eng.u()
            if not np.all(np.isfinite(out[s])):
                return None, float("nan")
    del keep
    return out, wall


def step_cost(lbmc, Lc, tau_c, model=None, c_smag=0.0, passes=2, steps=200):
    """Seconds per step of a coarse run (rest state, periodic, forced)."""
    n = Lc ** 3
    cfg = lbmc.make_config("d3q15", (Lc, Lc, Lc), tau=tau_c, collision_type=lbmc.BGK, forcing=True,
                           c_smag=c_smag)
    F = np.full((3, n), 1e-7)
    F[0, ::2] = 2e-7  # not uniform: the force is read per node, as in the study
    dom, keep = lbmc.make_domain(n, 3, 15, None, F)
    with lbmc.Engine(cfg, dom) as eng:
        if model is not None and model != "smag":
            model.attach(eng, iterations=passes)
        eng.iterate(20, lbmc.SYNC)
        best = float("inf")
        for _ in range(3):
            t = time.perf_counter()
            eng.iterate(steps, lbmc.SYNC)
            best = min(best, (time.perf_counter() - t) / steps)
    del keep
    return best


def spectrum(u, L):
    """Shell-summed kinetic-energy spectrum E(k), k = 1 .. L/2 - 1."""
    U = np.fft.fftn(u.reshape(3, L, L, L), axes=(1, 2, 3)) / L ** 3
    e = 0.5 * (np.abs(U) ** 2).sum(0)
    k = np.fft.fftfreq(L, 1.0 / L)
    kz, ky, kx = np.meshgrid(k, k, k, indexing="ij")
    kk = np.rint(np.sqrt(kx * kx + ky * ky + kz * kz)).astype(int)
    E = np.bincount(kk.reshape(-1), weights=e.reshape(-1), minlength=L)
    return E[1:L // 2]


def velocity_error(u_c, u_ref):
    return float(np.linalg.norm(u_c - u_ref) / np.linalg.norm(u_ref))


def spectrum_error(u_c, Lc, E_ref, kmax):
    """Mean |log E_c(k) - log E_ref(k)| over the shells k = 1 .. kmax."""
    Ec = spectrum(u_c, Lc)
    return float(np.mean(np.abs(np.log(Ec[:kmax] + 1e-300) - np.log(E_ref[:kmax] + 1e-300))))


def run_pipeline(lbmc, torch, L=256, factors=(4,), tau=0.51, amp=4e-6, kmax=2,
                 train_snaps=(12000, 14000, 16000, 18000), eval_start=16000,
                 eval_checks=(16200, 16500, 17000, 18000, 20000, 24000),
                 epochs=8, seed_train=1, seed_eval=2, log=print):
    """Learned-closure study; returns a dict of results per coarse factor.

    Per factor (coarse grid Lc = L / factor): training set from the box-
    filtered training solve, a-priori scores on a held-out snapshot, then
    coarse runs from the filtered evaluation snapshot at eval_start: no
    model, Smagorinsky (C_s = 0.1), the learned closure with 1 and 2
    fixed-point passes, and Smagorinsky on the finest grid whose measured
    wall clock stays within the learned run's (equal wall clock), started
    from the same coarse data Fourier-interpolated.  Errors: filtered
    velocity at each check time (a finer grid's field truncated to the
    coarse grid's Fourier modes first) and the energy spectrum against the
    fine solve's on shells k <= Lc / 4.
    """
    dev = torch.device("cuda")
    t0 = time.perf_counter()
    F_train = fourier_force(L, amp, kmax, seed_train)
    train = fine_solve(lbmc, L, tau, max(train_snaps), list(train_snaps), F_train)
    F_eval = fourier_force(L, amp, kmax, seed_eval)
    ev = fine_solve(lbmc, L, tau, max(eval_checks), [eval_start] + list(eval_checks), F_eval)
    log(f"fine solves done in {time.perf_counter() - t0:.1f} s")
    t_end = max(eval_checks)
    out = {"fine": {"L": L, "tau": tau, "amp": amp, "kmax": kmax,
                    "u_rms": {s: float(np.sqrt((ev[s][1] ** 2).mean())) for s in ev}}}
    nu_f = (tau - 0.5) / 3
    Ft = torch.as_tensor(F_eval, device=dev).reshape(3, L, L, L)
    E_fine = {s: spectrum(ev[s][1], L) for s in eval_checks[-2:]}
    for factor in factors:
        Lc = L // factor
        kcmp = Lc // 4
        X, y = dataset(lbmc, torch, [train[s] for s in train_snaps], L, factor, dev)
        t1 = time.perf_counter()
        model, hist = train_closure(lbmc, X, y, epochs=epochs)
        t_train = time.perf_counter() - t1
        res = {"coarse_L": Lc, "samples": int(len(y)), "train_s": t_train,
               "loss_first": float(hist[0]), "loss_last": float(hist[-1]),
               "nu_star_mean": float(y.mean()),
               "a_priori": a_priori(lbmc, torch, model, *ev[eval_start], L, factor, dev)}
        log(f"factor {factor} a priori: {res['a_priori']}")
        rb0, ub0, _ = filtered(torch, *ev[eval_start], L, factor, dev)
        refs = {s: filtered(torch, *ev[s], L, factor, dev)[1].cpu().numpy().reshape(3, -1)
                for s in eval_checks}

        def run(N, name, model_arg, cs, passes=2):
            """One coarse run on N^3 from the filtered data (interpolated if N != Lc)."""
            r0, u0 = rb0, ub0
            if N != Lc:
                r0 = fourier_resample(torch, rb0[None], N)[0]
                u0 = fourier_resample(torch, ub0, N)
            Fc = (L / N) * fourier_resample(torch, Ft, N).reshape(3, -1).cpu().numpy()
            tau_c = 0.5 + 3 * nu_f * N / L
            checks = {s: int(round((s - eval_start) * N / L)) for s in eval_checks}
            snaps, wall = coarse_solve(lbmc, r0.cpu().numpy(), u0.cpu().numpy(), Fc, tau_c,
                                       sorted(set(checks.values())), model_arg, cs, passes)
            r = {"N": N, "tau": tau_c, "steps": checks[t_end], "wall_s": wall}
            if snaps is None:
                r["blew_up"] = True
            else:
                r["blew_up"] = False
                if N == Lc:
                    r["velocity_error"] = {s: velocity_error(snaps[checks[s]], refs[s]) for s in eval_checks}
                else:
                    # a finer grid: its field truncated to the coarse grid's
                    # Fourier modes, then compared like the others
                    r["velocity_error"] = {
                        s: velocity_error(
                            fourier_resample(torch, torch.as_tensor(snaps[checks[s]], device=dev)
                                             .reshape(3, N, N, N), Lc).reshape(3, -1).cpu().numpy(),
                            refs[s])
                        for s in eval_checks}
                r["spectrum_error"] = {s: spectrum_error(snaps[checks[s]], N, E_fine[s], kcmp)
                                       for s in E_fine}
            log(f"factor {factor} {name}: {r}")
            return r
        res["none"] = run(Lc, "none", None, 0.0)
        res["smagorinsky"] = run(Lc, "smagorinsky", "smag", 0.1)
        res["learned_1pass"] = run(Lc, "learned_1pass", model, 0.1, passes=1)
        res["learned_2pass"] = run(Lc, "learned_2pass", model, 0.1, passes=2)
        # Equal wall clock: the finest Smagorinsky grid (multiples of 8)
        # whose measured run time stays within the learned (1-pass) run's.
        c_learn = step_cost(lbmc, Lc, 0.5 + 3 * nu_f / factor, model, 0.1, passes=1)
        budget = c_learn * (t_end - eval_start) / factor
        best = Lc
        for N in range(Lc + 8, 2 * Lc + 1, 8):
            c = step_cost(lbmc, N, 0.5 + 3 * nu_f * N / L, "smag", 0.1)
            if c * (t_end - eval_start) * N / L <= budget:
                best = N
            else:
                break
        res["equal_wall_clock"] = {"learned_s_per_step": c_learn, "grid": best}
        res["smagorinsky_equal_wall_clock"] = run(best, "smagorinsky_equal_wall_clock", "smag", 0.1)
        out[f"factor{factor}"] = res
        model.close()
    return out
