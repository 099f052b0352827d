"""Learned subgrid closure: kernels checked against the FP64 CPU oracle.

- features: the device feature function vs oracle/mlp_oracle.py;
- gradients: GPU forward/backward (BF16 weights, FP32 accumulation) vs the
  FP64 numpy gradient with the same BF16-rounded weights;
- training: the GPU Adam loop fits a smooth target;
- in-step inference (warp-wide on the tensor cores, BF16 inputs and
  activations, FP32 accumulation) vs the oracle's emulation of those
  numerics, and every weight in its fragment slot, through
  lbmc_mlp_predict_step;
- the closure inside the step: D3Q15/D2Q9 BGK+Guo steps with the closure
  attached vs the restatement driven by per-node tau computed in numpy from
  the same populations; with an empty training range every node falls back
  to Smagorinsky and the step equals the Smagorinsky step.
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


def _normalised(feats, mean, std):
    """The step's FP32 normalisation fma(raw, 1/std, -mean/std)."""
    inv = np.float32(1) / np.asarray(std, np.float32)
    shift = -np.asarray(mean, np.float32) * inv
    x = feats.astype(np.float32).astype(np.float64) * inv.astype(np.float64) + shift.astype(np.float64)
    return x.astype(np.float32).astype(np.float64)


def test_step_inference_matches_oracle(lbmc):
    """The tensor-core evaluation the step uses vs the FP64 emulation of its
    BF16 numerics (oracle forward_step), and vs the FP32-activation network."""
    rng = np.random.default_rng(6)
    m, feats = _net(lbmc, rng, seed=9)
    y_tc = m.predict_step(feats).astype(np.float64) / 1e-3
    y_32 = m.predict(feats).astype(np.float64) / 1e-3
    xn = _normalised(feats, m._norm[0], m._norm[1])
    y_em = mo.forward_step(m.params().astype(np.float64), xn)
    scale = np.std(y_em)
    d_em, d_32 = np.abs(y_tc - y_em), np.abs(y_tc - y_32)
    print(f"in-step vs BF16 emulation: max {d_em.max() / scale:.2e} mean {d_em.mean() / scale:.2e};"
          f" vs FP32 activations: max {d_32.max() / scale:.2e} mean {d_32.mean() / scale:.2e} (x std)")
    # The hardware tanh (BF16, within one BF16 step of tanh) and the tensor
    # cores' accumulation order move single activations by one BF16 step
    # against the emulation; the pinning of every weight to its place is
    # test_step_inference_fragment_map's job.
    assert d_em.max() <= 0.1 * scale and d_em.mean() <= 1e-2 * scale
    # BF16 activations against the FP32-activation forward used in training.
    assert d_32.mean() <= 2e-2 * scale


def test_step_inference_fragment_map(lbmc):
    """Every weight in its fragment slot: with W2 a permutation, b2 = 0 and W3
    the unit vector e_k, the output is hidden unit pi(k) of layer 1 through
    both SiLUs, y = silu_b(silu_b(W1[pi(k)] x + b1[pi(k)])) + b3.  The biases
    keep every pre-activation positive, where the BF16 SiLU is within one
    BF16 step of the emulation (in the negative tail h + h tanh(h) cancels
    and the hardware tanh's last bit dominates), so for each of the 32 k the
    output must equal the emulation to within three BF16 steps."""
    rng = np.random.default_rng(8)
    m = lbmc.Mlp(seed=2)
    S, rho = random_strain(2000, rng)
    feats = mo.strain_features(S, rho)
    m.set_normalization(feats.mean(0), feats.std(0), target_scale=1.0)
    xn = _normalised(feats, m._norm[0], m._norm[1])
    perm = rng.permutation(mo.H)
    base = np.zeros(mo.PARAMS)
    base[mo.W1:mo.B1] = 0.3 * rng.standard_normal(mo.H * mo.IN)
    base[mo.B1:mo.W2] = 8.0 + rng.uniform(0, 2, mo.H)
    base[mo.W2:mo.B2] = np.eye(mo.H)[perm].reshape(-1)
    base[mo.B3] = 0.25
    exact = []
    for k in range(mo.H):
        p = base.copy()
        p[mo.W3 + k] = 1.0
        m.set_params(p)
        y_tc = m.predict_step(feats).astype(np.float64)
        y_em = mo.forward_step(m.params().astype(np.float64), xn)
        a = y_em - 0.25  # the selected activation, > 0
        assert a.min() > 1.0
        step = 2.0 ** (np.floor(np.log2(a)) - 7)
        assert np.all(np.abs(y_tc - y_em) <= 3 * step), (k, np.max(np.abs(y_tc - y_em) / step))
        exact.append(np.mean(y_tc == y_em))
    assert np.mean(exact) >= 0.8, np.mean(exact)


def numpy_tau(f, lattice, F, tau0, c_smag, nu_net, norm, iterations):
    """Per-node tau of the closure (with Smagorinsky fallback), FP64; the
    network value nu_net(raw features) = target_scale * y."""
    e, w = E[lattice].astype(np.float64), W[lattice]
    rho = f.sum(0)
    u = (e @ f) / rho
    if F is not None:
        u = u + np.asarray(F)[:, None] / (2 * rho)
    eu = 3 * (e.T @ u)
    feq = rho * w[:, None] * (1 + eu + 0.5 * eu * eu - 1.5 * (u * u).sum(0))
    neq = f - feq
    ex, ey, ez = np.vstack([e, np.zeros((3 - e.shape[0], e.shape[1]))])
    q = np.stack([(ex * ex) @ neq, (ey * ey) @ neq, (ez * ez) @ neq,
                  (ex * ey) @ neq, (ey * ez) @ neq, (ex * ez) @ neq], 1)
    r2 = np.sqrt(2.0)
    qhat = r2 * (np.abs(q[:, :3]).sum(1) + 2 * np.abs(q[:, 3:]).sum(1))
    k = 2 * r2 * c_smag ** 2 * (9 / rho)
    tau_smag = tau0 + 0.5 * (np.sqrt(tau0 ** 2 + k * qhat) - tau0)
    mean, std, lo, hi = norm
    tau = tau_smag.copy()  # the fixed point starts from the Smagorinsky tau
    ok = np.ones(len(rho), bool)
    for _ in range(iterations):
        S = -1.5 * q / (rho * tau)[:, None]
        raw = mo.strain_features(S, rho)
        x = (raw - mean) / std
        ok &= np.all((x >= lo) & (x <= hi), 1)
        tau = np.where(ok, tau0 + 3 * np.maximum(0.0, nu_net(np.where(ok[:, None], raw, mean))), tau)
    return np.where(ok, tau, tau_smag)


# (12, 10, 8): one partly filled warp per row; (40, 6, 5) with solids: solid
# lanes and a second warp with 8 active lanes; D2Q9 the 2-D strain path.
# net "const": W1 = W2 = 0, so nu_t is one value wherever the inputs are in
# range and the step must match to rounding; "fallback": nothing in range,
# the step equals the Smagorinsky step; "random": a random network.
CLOSURE_CASES = [("d3q15", (12, 10, 8), 0.0, "const"), ("d3q15", (40, 6, 5), 0.2, "const"),
                 ("d2q9", (70, 9, 1), 0.15, "const"), ("d3q15", (12, 10, 8), 0.0, "fallback"),
                 ("d3q15", (12, 10, 8), 0.0, "random"), ("d3q15", (40, 6, 5), 0.2, "random"),
                 ("d2q9", (70, 9, 1), 0.15, "random")]


@pytest.mark.parametrize("lattice,length,solids,net", CLOSURE_CASES)
def test_closure_step_matches_oracle(lbmc, lattice, length, solids, net):
    """The closure inside the step: strain estimate, features, range check,
    fixed point from the Smagorinsky tau, fallback, and warp participation of
    solid and out-of-range lanes, against numpy; the network value comes from
    the step's own evaluator (lbmc_mlp_predict_step), which the two tests
    above pin to the oracle."""
    rng = np.random.default_rng(4)
    case = make_case(lattice, length, 0, True, solids=solids, seed=5, uniform_force=True, u_amp=0.05)
    case.c_smag = 0.1
    case.tau = 0.52
    m = lbmc.Mlp(seed=11)
    p = 0.3 * rng.standard_normal(mo.PARAMS)
    if net == "const":
        p[mo.W1:mo.B1] = 0.0
        p[mo.W2:mo.B2] = 0.0
        p[mo.B3] = 2.0
    m.set_params(p)
    # Normalisation from the case's own strain field, so the inputs are O(1).
    ref = Restatement(case)
    with np.errstate(all="ignore"):
        feats = _case_features(ref.f(), lattice, case.force[:, 0], case.tau)
    fluid = np.all(np.isfinite(feats), 1) & (case.geometry.reshape(-1) == 0)
    mean, std = feats[fluid].mean(0), feats[fluid].std(0)
    std = np.where(std > 0, std, 1.0)  # 2-D: det S = 0
    if net == "fallback":
        lo, hi = np.full(6, 1e29), np.full(6, 1e30)  # nothing is in range
    else:
        lo, hi = np.full(6, -1e30), np.full(6, 1e30)
    m.set_normalization(mean, std, lo, hi, target_scale=3e-3)
    norm = (m._norm[0].astype(np.float64), m._norm[1].astype(np.float64), lo, hi)
    F = case.force[:, 0]
    steps, iters = 6, 2
    with lbmc.Engine.from_case(case, storage=lbmc.F64) as eng:
        m.attach(eng, iterations=iters)
        eng.iterate(steps, lbmc.SYNC)
        f_gpu = eng.f()

    def nu_net(raw):
        return m.predict_step(raw).astype(np.float64)
    for _ in range(steps):
        with np.errstate(all="ignore"):  # solid nodes: their tau is never used
            tau = numpy_tau(ref.f(), lattice, F, case.tau, case.c_smag, nu_net, norm, iters)
        ref.set_tau_field(np.where(np.isfinite(tau), tau, case.tau))
        ref.run(1)
    err = np.abs(f_gpu - ref.f()).max() / np.abs(ref.f()).max()
    print(f"{lattice} {length} {net}: max |f_gpu - f_oracle| / max |f| = {err:.2e}")
    if net == "random":
        # The GPU computes the features in FP32 (the trace and det S are
        # ill-conditioned), this side in FP64: where that flips the BF16
        # rounding of an input, nu_t moves by ~1e-5 at that node and step.
        assert err <= 2e-4, err
    else:
        assert err <= 1e-12, err
    if net == "fallback":
        with lbmc.Engine.from_case(case, storage=lbmc.F64) as eng:
            eng.iterate(steps, lbmc.SYNC)
            np.testing.assert_allclose(eng.f(), f_gpu, rtol=0, atol=1e-15)


def _case_features(f, lattice, F, tau0):
    """Raw closure features of a population field at tau = tau0."""
    e, w = E[lattice].astype(np.float64), W[lattice]
    rho = f.sum(0)
    u = (e @ f) / rho + np.asarray(F)[:, None] / (2 * rho)
    eu = 3 * (e.T @ u)
    neq = f - rho * w[:, None] * (1 + eu + 0.5 * eu * eu - 1.5 * (u * u).sum(0))
    ex, ey, ez = np.vstack([e, np.zeros((3 - e.shape[0], e.shape[1]))])
    q = np.stack([(ex * ex) @ neq, (ey * ey) @ neq, (ez * ez) @ neq,
                  (ex * ey) @ neq, (ey * ez) @ neq, (ex * ez) @ neq], 1)
    return mo.strain_features(-1.5 * q / (rho * tau0)[:, None], rho)
