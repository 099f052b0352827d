"""AA-pattern streaming (LBMC_STREAM_AA) against the shift layout.

The two layouts hold the same state after every step; only the slot a
value sits in differs (even steps read and write each node's own slots,
odd steps its neighbours').  AA runs in the tiled layout (64-node tiles,
populations of a tile back to back) when Lx is a multiple of 64 and in the
plain AA layout otherwise; both are covered.  So every result read through the public API
must be bit-identical: populations (natural order, un-mapped by
lbmc_fetch), stored rho/u and the FP64 diagnostic sums, after odd and
even step counts, for every collision type, forcing, macro, Zou-He and
stress-free boundaries, partial solids, both lattices, FP64/FP32/FP16
storage (FP16 also with stochastic rounding, whose random bits depend on
node, step and population only), and the learned closure in FP64 (its FP32 kernels agree to the
FP32 rounding level).  The shift layout is itself checked
against the oracle (test_parity_gpu.py), which pins AA to it as well.
"""
import numpy as np
import pytest

from cases import make_case

pytestmark = pytest.mark.gpu

AA_COMBOS = [(lat, ct, forcing, bc, smag)
             for lat in ("d2q9", "d3q15") for ct in range(4) for forcing in (False, True)
             for bc in (None, "random", "zh", "sf") for smag in (0.0, 0.1) if not (smag and ct >= 2)]


def run(lbmc, case, steps, storage, streaming):
    with lbmc.Engine.from_case(case, storage=lbmc.STORAGE_IDS[storage], streaming=streaming) as eng:
        out = []
        done = 0
        for s in steps:
            eng.iterate(s - done, lbmc.STORE_MACROS | lbmc.REDUCE_DIAG | lbmc.SYNC)
            done = s
            d = eng.diag()
            out.append((eng.f(), eng.rho(), eng.u(),
                        np.array([d.mass, *d.momentum, d.kinetic_energy])))
        return out


LENGTHS = {("d2q9", False): (37, 21, 1), ("d3q15", False): (19, 11, 9),
           ("d2q9", True): (128, 9, 1), ("d3q15", True): (64, 7, 6)}


@pytest.mark.parametrize("tiled", [False, True], ids=["plain", "tiled"])
@pytest.mark.parametrize("storage", ["f32", "f16", "f16sr", "f64"])
@pytest.mark.parametrize("lat,ct,forcing,bc,smag", AA_COMBOS)
def test_aa_equals_shift(lbmc, lat, ct, forcing, bc, smag, storage, tiled):
    if storage != "f32" and (forcing or smag or ct in (1, 2)):
        pytest.skip("storage formats are covered on the plain and MRT+partial cases")
    length = LENGTHS[(lat, tiled)]
    case = make_case(lat, length, ct, forcing, solids=0.08, partial=0.15 if ct % 2 else 0.0,
                     macro="random" if bc == "random" else None,
                     micro=bc if bc in ("zh", "sf") else None, c_smag=smag, seed=7 + ct)
    steps = [1, 2, 7, 20]
    a = run(lbmc, case, steps, storage, lbmc.STREAM_SHIFT)
    b = run(lbmc, case, steps, storage, lbmc.STREAM_AA)
    for x, y in zip(a, b):
        for p, q in zip(x, y):
            np.testing.assert_array_equal(p, q)


def test_aa_large_periodic_and_closure(lbmc):
    """A 64^3 periodic forced box (every block, ragged-free) and the learned
    closure's warp-wide path under AA."""
    rng = np.random.default_rng(3)
    case = make_case("d3q15", (64, 64, 64), 0, True, seed=2, uniform_force=True, u_amp=0.03)
    case.c_smag = 0.1
    a = run(lbmc, case, [5, 10], "f32", lbmc.STREAM_SHIFT)
    b = run(lbmc, case, [5, 10], "f32", lbmc.STREAM_AA)
    for x, y in zip(a, b):
        for p, q in zip(x, y):
            np.testing.assert_array_equal(p, q)
    m = lbmc.Mlp(seed=4)
    m.set_params(0.3 * rng.standard_normal(1313))
    m.set_normalization(np.zeros(6), np.full(6, 5.0), target_scale=1e-3)
    for length in ((40, 6, 5), (64, 6, 5)):  # plain and tiled AA layout
        _closure_aa_vs_shift(lbmc, m, length)
    m.close()


def _closure_aa_vs_shift(lbmc, m, length):
    small = make_case("d3q15", length, 0, True, solids=0.2, seed=5, uniform_force=True)
    small.c_smag = 0.1
    for storage in (lbmc.F64, lbmc.F32):
        res = []
        for streaming in (lbmc.STREAM_SHIFT, lbmc.STREAM_AA):
            with lbmc.Engine.from_case(small, storage=storage, streaming=streaming) as eng:
                m.attach(eng, iterations=2)
                eng.iterate(9, lbmc.SYNC)
                res.append(eng.f())
        if storage == lbmc.F64:
            np.testing.assert_array_equal(res[0], res[1])
        else:
            # Each run is deterministic, but the FP32 closure kernels of the
            # two layouts are separate instantiations whose FP32 arithmetic
            # the compiler contracts differently: differences at the FP32
            # rounding level appear from the first odd step on.
            assert np.abs(res[0] - res[1]).max() <= 1e-7 * np.abs(res[0]).max()


def test_aa_rejects_pipelined_kernel(lbmc):
    case = make_case("d3q15", (24, 8, 8), seed=1)
    with pytest.raises(lbmc.LbmcError) as ei:
        lbmc.Engine.from_case(case, streaming=lbmc.STREAM_AA, kernel=lbmc.KERNEL_PIPELINED)
    assert ei.value.status == lbmc.ERR_UNSUPPORTED
