"""Batched persistent launch (lbmc_batch_*): every domain must evolve exactly
as the single-domain step does.  Compared per domain against the FP64
restatement (FP32 storage: err <= 1e-5; FP16: <= 5e-3), with domains that
stay in shared memory and domains that are stepped in HBM in the same batch,
and with the autotuned launch shape."""
import numpy as np
import pytest

from oracle.oracle import Case, Restatement

pytestmark = pytest.mark.gpu

TAU = 0.9
FORCE = (2e-5, -5e-6)


def domains(seed=3):
    import workloads
    rng = np.random.default_rng(seed)
    shapes = [(16, 24), (40, 33), (96, 120), (75, 160), (33, 64), (130, 90), (90, 200)]
    return [workloads.circle_domain(lx, ly, rng.uniform(0.2, 0.4), rng, tau=TAU)
            for ly, lx in shapes]


def reference(geom, steps):
    ly, lx = geom.shape
    n = lx * ly
    force = np.zeros((2, n))
    force[0], force[1] = FORCE
    case = Case(lattice="d2q9", length=(lx, ly, 1), tau=TAU, collision_type=1, forcing=True,
                geometry=geom.reshape(n), force=force)
    r = Restatement(case)
    r.run(steps)
    return r.f()


def err(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


@pytest.mark.parametrize("storage,tol,threads,spl", [
    ("f32", 1e-5, 512, 8), ("f32", 1e-5, 0, 0), ("f16", 5e-3, 256, 16), ("bf16", 3e-2, 1024, 4)])
def test_batch_matches_single_domain_oracle(lbmc, storage, tol, threads, spl):
    geoms = domains()
    steps = 37
    with lbmc.Batch(geoms, tau=TAU, force=FORCE, collision_type=lbmc.NTPOR, storage=storage,
                    block_threads=threads, steps_per_launch=spl) as b:
        res = b.run(steps, 0.0, check_every=5)
        info = b.info()
        assert 0 < info["resident_domains"] < len(geoms)
        for d, g in enumerate(geoms):
            assert res[d].steps == steps
            assert err(b.fetch(d, lbmc.FIELD_F), reference(g, steps)) <= tol


def test_batch_converges_and_freezes(lbmc):
    geoms = domains(seed=9)[:4]
    with lbmc.Batch(geoms, tau=1.0, force=(1e-6, 0.0), storage="f32") as b:
        res = b.run(200000, 1e-9, check_every=50)
        for d in range(len(geoms)):
            assert res[d].converged == 1
            assert res[d].delta_u < 1e-9
            assert res[d].elapsed_ms > 0
        f1 = [b.fetch(d, lbmc.FIELD_F) for d in range(len(geoms))]
        again = b.run(200000, 1e-9, check_every=50)  # converged domains stay frozen
        for d in range(len(geoms)):
            assert again[d].steps == res[d].steps
            np.testing.assert_array_equal(b.fetch(d, lbmc.FIELD_F), f1[d])


# FP16's quantisation floor of max|u(t) - u(t - C)| is above 1e-9: a
# tolerance above it lets its domains converge too.
@pytest.mark.parametrize("storage,tol,cap", [("f32", 1e-9, 200000), ("f16", 1e-5, 50000)])
def test_batch_tail_phase_is_bit_identical(lbmc, storage, tol, cap):
    """The wide path (HBM domains spread over every SM, one step per launch,
    segments rebuilt as domains stop) and the one-block-per-domain path run
    the same node update and the same convergence rule, so a batch run to
    steady state ends bit for bit the same (step counts, convergence, last
    delta_u and populations) whichever path each HBM domain takes: all one
    block per domain, all wide, split by size (12000 nodes: two of the four
    HBM domains each way), the storage's default split, and block-stepped
    domains that join the wide path once fewer than 3 of them are left."""
    geoms = domains()
    runs = []
    for wide_min, wide_below in ((1 << 30, -1), (1, -1), (12000, -1), (0, 0), (1 << 30, 3)):
        with lbmc.Batch(geoms, tau=1.0, force=(1e-6, 0.0), collision_type=lbmc.NTPOR, storage=storage,
                        block_threads=256, steps_per_launch=50, wide_below=wide_below,
                        wide_min_nodes=wide_min) as b:
            res = b.run(cap, tol, check_every=50)
            runs.append(([(r.steps, r.converged, r.delta_u) for r in res],
                         [b.fetch(d, lbmc.FIELD_F) for d in range(len(geoms))]))
    steps = [r[0] for r in runs[0][0]]
    assert len(set(steps)) >= 2  # domains converge at different times
    for other in runs[1:]:
        assert other[0] == runs[0][0]
        for x, y in zip(runs[0][1], other[1]):
            np.testing.assert_array_equal(x, y)


@pytest.mark.parametrize("storage,wide_below", [("f32", -1), ("f32", 100), ("f16", -1)])
@pytest.mark.parametrize("wide_min", [1 << 30, 1])
def test_batch_nonfinite_domain_is_reported(lbmc, storage, wide_below, wide_min):
    """A domain whose velocity turns non-finite is stopped and flagged, not
    taken for converged (a max that drops NaN would read it as Delta u = 0).
    The planted fault is on the host: a negative porosity patch in one
    domain kept in shared memory and one stepped in HBM, which the
    Noble-Torczynski blend amplifies until the populations overflow.
    wide_below = 100 moves the block-stepped HBM domains to the wide path at
    once; wide_min = 1 puts every HBM domain there from the start."""
    geoms = [g.copy() for g in domains(seed=9)[:4]]
    for d in (1, 3):
        geoms[d][2:6, 2:6] = -50.0
    with lbmc.Batch(geoms, tau=1.0, force=(1e-6, 0.0), storage=storage,
                    wide_below=wide_below, wide_min_nodes=wide_min) as b:
        if storage == "f32":  # FP16 rows are half as long: all four fit in shared memory
            assert b.info()["resident_domains"] == 2
        with pytest.raises(lbmc.LbmcError) as ei:
            b.run(3000, 1e-12, check_every=50)
        assert ei.value.status == lbmc.ERR_NAN
        res = ei.value.results
        for d in range(4):
            if d in (1, 3):
                assert res[d].nonfinite == 1 and res[d].converged == 0
                assert np.isnan(res[d].delta_u)
                assert res[d].steps < 3000 and res[d].elapsed_ms == -1.0
            else:
                # small FP32 domains may reach an exact fixed point (delta_u = 0)
                assert res[d].nonfinite == 0 and np.isfinite(res[d].delta_u)
                assert res[d].converged == 1 or res[d].steps == 3000
