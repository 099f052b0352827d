"""Learned subgrid closure: kernels checked against the FP64 CPU oracle.

- features: the device feature function vs oracle/mlp_oracle.py;
- gradients: GPU forward/backward (BF16 weights, FP32 accumulation) vs the
  FP64 numpy gradient with the same BF16-rounded weights;
- training: the GPU Adam loop fits a smooth target;
- inference inside the step: a D3Q15 BGK+Guo step with the closure attached
  vs the restatement driven by per-node tau computed in numpy from the same
  populations; with an empty training range every node falls back to
  Smagorinsky and the step equals the Smagorinsky step.
"""
import numpy as np
import pytest

from cases import E, W, make_case
from oracle import mlp_oracle as mo
from oracle.oracle import Restatement

pytestmark = pytest.mark.gpu


def random_strain(n, rng, scale=1e-3):
    S = rng.standard_normal((n, 6)) * scale * np.exp(rng.uniform(-3, 1, (n, 1)))
    return S, 1 + 0.01 * rng.standard_normal(n)


def test_features_match_oracle(lbmc):
    rng = np.random.default_rng(0)
    S, rho = random_strain(5000, rng)
    f_gpu = lbmc.mlp_features(S, rho)
    f_cpu = mo.strain_features(S.astype(np.float32), rho.astype(np.float32))
    np.testing.assert_allclose(f_gpu, f_cpu, rtol=2e-5, atol=2e-4)


def _net(lbmc, rng, seed=3):
    m = lbmc.Mlp(seed=seed)
    p = rng.standard_normal(mo.PARAMS) * 0.3
    m.set_params(p)
    S, rho = random_strain(20000, rng)
    feats = mo.strain_features(S, rho)
    m.set_normalization(feats.mean(0), feats.std(0), target_scale=1e-3)
    return m, feats


def test_gradients_match_cpu_oracle(lbmc):
    rng = np.random.default_rng(1)
    m, feats = _net(lbmc, rng)
    X = feats[:3000]
    t = 1e-3 * rng.standard_normal(3000)
    g_gpu, loss_gpu = m.gradients(X, t)
    mean, std = m._norm[0].astype(np.float64), m._norm[1].astype(np.float64)
    xn = (X.astype(np.float32).astype(np.float64) - mean) / std
    loss_cpu, g_cpu = mo.loss_and_grad(m.params().astype(np.float64), xn, t / 1e-3)
    assert abs(loss_gpu - loss_cpu) <= 1e-4 * loss_cpu
    assert np.linalg.norm(g_gpu - g_cpu) <= 1e-4 * np.linalg.norm(g_cpu)


def test_training_fits_smooth_target(lbmc):
    rng = np.random.default_rng(2)
    m, feats = _net(lbmc, rng, seed=7)
    m.set_params(lbmc.Mlp(seed=7).params())  # Xavier start
    xn = (feats - feats.mean(0)) / feats.std(0)
    target = 1e-3 * (0.5 * np.tanh(xn[:, 0]) + 0.3 * xn[:, 1] ** 2 / (1 + xn[:, 1] ** 2))
    hist = m.train(feats, target, epochs=30, batch=512, lr=3e-3)
    assert hist[-1] < 0.05 * hist[0]
    pred = m.predict(feats)
    assert np.sqrt(np.mean((pred - target) ** 2)) < 0.1 * np.std(target)


def numpy_tau(f, lattice, F, tau0, c_smag, params, norm, iterations):
    """Per-node tau of the closure (with Smagorinsky fallback), FP64."""
    e, w = E[lattice].astype(np.float64), W[lattice]
    rho = f.sum(0)
    u = (e @ f) / rho
    if F is not None:
        u = u + np.asarray(F)[:, None] / (2 * rho)
    eu = 3 * (e.T @ u)
    feq = rho * w[:, None] * (1 + eu + 0.5 * eu * eu - 1.5 * (u * u).sum(0))
    neq = f - feq
    ex, ey, ez = e
    q = np.stack([(ex * ex) @ neq, (ey * ey) @ neq, (ez * ez) @ neq,
                  (ex * ey) @ neq, (ey * ez) @ neq, (ex * ez) @ neq], 1)
    r2 = np.sqrt(2.0)
    qhat = r2 * (np.abs(q[:, :3]).sum(1) + 2 * np.abs(q[:, 3:]).sum(1))
    k = 2 * r2 * c_smag ** 2 * (9 / rho)
    tau_smag = tau0 + 0.5 * (np.sqrt(tau0 ** 2 + k * qhat) - tau0)
    mean, std, lo, hi, scale = norm
    tau = np.full(len(rho), tau0)
    ok = np.ones(len(rho), bool)
    for _ in range(iterations):
        S = -1.5 * q / (rho * tau)[:, None]
        x = (mo.strain_features(S, rho) - mean) / std
        ok &= np.all((x >= lo) & (x <= hi), 1)
        y, _ = mo.forward(params, x)
        tau = np.where(ok, tau0 + 3 * np.maximum(0.0, scale * y), tau)
    return np.where(ok, tau, tau_smag)


@pytest.mark.parametrize("mode", ["learned", "fallback"])
def test_closure_step_matches_oracle(lbmc, mode):
    rng = np.random.default_rng(4)
    case = make_case("d3q15", (12, 10, 8), 0, True, seed=5, uniform_force=True, u_amp=0.05)
    case.c_smag = 0.1
    case.tau = 0.52
    m = lbmc.Mlp(seed=11)
    m.set_params(0.2 * rng.standard_normal(mo.PARAMS))
    S, rho = random_strain(4000, rng, scale=3e-3)
    feats = mo.strain_features(S, rho)
    mean, std = feats.mean(0), feats.std(0)
    if mode == "learned":
        lo, hi = np.full(6, -1e30), np.full(6, 1e30)
    else:
        lo, hi = np.full(6, 1e29), np.full(6, 1e30)  # nothing is in range
    m.set_normalization(mean, std, lo, hi, target_scale=1e-2)
    norm = (m._norm[0].astype(np.float64), m._norm[1].astype(np.float64), lo, hi, 1e-2)
    params = m.params().astype(np.float64)
    F = case.force[:, 0]
    steps, iters = 6, 2
    with lbmc.Engine.from_case(case, storage=lbmc.F64) as eng:
        m.attach(eng, iterations=iters)
        eng.iterate(steps, lbmc.SYNC)
        f_gpu = eng.f()
    ref = Restatement(case)
    for _ in range(steps):
        ref.set_tau_field(numpy_tau(ref.f(), "d3q15", F, case.tau, case.c_smag, params, norm, iters))
        ref.run(1)
    err = np.abs(f_gpu - ref.f()).max() / np.abs(ref.f()).max()
    assert err <= 1e-6
    if mode == "fallback":
        with lbmc.Engine.from_case(case, storage=lbmc.F64) as eng:
            eng.iterate(steps, lbmc.SYNC)
            np.testing.assert_allclose(eng.f(), f_gpu, rtol=0, atol=1e-15)
