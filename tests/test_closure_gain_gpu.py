"""What the learned closure gains, at test scale, through the same pipeline
as the full study (lbm-c_b200/closure.py): a forced-turbulence fine solve
on 64^3 (D3Q15 BGK, tau 0.51), box filter x4 to 16^3, the least-squares
eddy viscosity nu* as target, training on one solve, scoring on an
independent one (other forcing seed).  On the held-out filtered field the
learned nu_t, as the step evaluates it (tensor cores, Smagorinsky outside
the training range), must track nu* better than Smagorinsky's
C_s^2 |S| does: higher correlation and lower error of the subgrid
dissipation 2 nu_t S:S; and a coarse run with it must stay finite.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

L, FACTOR, TAU, AMP = 64, 4, 0.51, 1.6e-5


@pytest.fixture(scope="module")
def study(lbmc):
    import torch
    import closure
    dev = torch.device("cuda")
    snaps = (3000, 3500, 4000, 4500, 5000, 5500)
    train = closure.fine_solve(lbmc, L, TAU, max(snaps), list(snaps),
                               closure.fourier_force(L, AMP, 2, seed=1))
    F_eval = closure.fourier_force(L, AMP, 2, seed=2)
    ev = closure.fine_solve(lbmc, L, TAU, 5000, [4000, 5000], F_eval)
    X, y = closure.dataset(lbmc, torch, [train[s] for s in snaps], L, FACTOR, dev)
    model, hist = closure.train_closure(lbmc, X, y, epochs=40, batch=1024, lr=3e-3)
    yield dict(torch=torch, closure=closure, dev=dev, train=train, ev=ev, F_eval=F_eval,
               model=model, hist=hist, X=X, y=y)
    model.close()


def test_fine_solve_is_turbulent_and_finite(study):
    u = study["ev"][5000][1]
    assert np.all(np.isfinite(u))
    u_rms = np.sqrt((u ** 2).mean())
    print(f"u_rms {u_rms:.4f}")
    assert 0.01 < u_rms < 0.15


def test_learned_nu_beats_smagorinsky_a_priori(study, lbmc):
    hist = study["hist"]
    assert hist[-1] < hist[0]
    s = study["closure"].a_priori(lbmc, study["torch"], study["model"], *study["ev"][5000], L, FACTOR,
                                  study["dev"])
    print(s)
    assert s["inside_range"] > 0.9
    assert s["learned"]["corr"] > s["smagorinsky"]["corr"] + 0.05
    assert s["learned"]["dissipation_rel_l2"] < s["smagorinsky"]["dissipation_rel_l2"]


def test_coarse_run_with_learned_closure_stays_finite(study, lbmc):
    torch, closure = study["torch"], study["closure"]
    Lc = L // FACTOR
    rb, ub, _ = closure.filtered(torch, *study["ev"][4000], L, FACTOR, study["dev"])
    Fc = FACTOR * np.stack([study["F_eval"][d].reshape(Lc, FACTOR, Lc, FACTOR, Lc, FACTOR)
                            .mean(axis=(1, 3, 5)).reshape(-1) for d in range(3)])
    tau_c = 0.5 + (TAU - 0.5) / FACTOR
    rbn, ubn = rb.cpu().numpy(), ub.cpu().numpy()
    none, _ = closure.coarse_solve(lbmc, rbn, ubn, Fc, tau_c, [250], None, 0.0)
    learned, _ = closure.coarse_solve(lbmc, rbn, ubn, Fc, tau_c, [250], study["model"], 0.1, passes=1)
    print("unclosed coarse run:", "non-finite" if none is None else "finite")
    assert learned is not None and np.all(np.isfinite(learned[250]))
