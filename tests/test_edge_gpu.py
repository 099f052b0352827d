"""Edge cases of the step: degenerate axes (L = 1, 2: the periodic wrap
lands on the node itself or its only neighbour), rows longer than one block
with a partly filled last block, and the shortest calls, all against the
FP64 restatement, in the shift and AA layouts."""
import numpy as np
import pytest

from cases import make_case
from oracle.oracle import Restatement

pytestmark = pytest.mark.gpu

TINY = [("d3q15", (1, 1, 1)), ("d3q15", (1, 7, 5)), ("d3q15", (2, 1, 3)), ("d3q15", (3, 2, 1)),
        ("d2q9", (1, 1, 1)), ("d2q9", (1, 6, 1)), ("d2q9", (2, 2, 1)), ("d2q9", (5, 1, 1)),
        # whole 64-node tiles along x: the tiled AA layout, one tile per row
        ("d3q15", (64, 1, 1)), ("d3q15", (64, 2, 1)), ("d3q15", (64, 1, 3)), ("d2q9", (64, 1, 1))]


def err(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


def run_both(lbmc, case, steps, storage, streaming):
    with lbmc.Engine.from_case(case, storage=storage, streaming=streaming) as eng:
        eng.iterate(steps, lbmc.STORE_MACROS | lbmc.SYNC)
        f = eng.f()
    ref = Restatement(case)
    ref.run(steps)
    return f, ref.f()


@pytest.mark.parametrize("streaming", ["shift", "aa"])
@pytest.mark.parametrize("lat,length", TINY)
def test_degenerate_axes(lbmc, lat, length, streaming):
    case = make_case(lat, length, 2 if lat == "d3q15" else 0, True, seed=4)
    sm = lbmc.STREAM_AA if streaming == "aa" else lbmc.STREAM_SHIFT
    for steps in (1, 2, 9):
        f, r = run_both(lbmc, case, steps, lbmc.F64, sm)
        assert err(f, r) <= 1e-10, (steps, err(f, r))


@pytest.mark.parametrize("streaming", ["shift", "aa"])
@pytest.mark.parametrize("lat,length,ct,bc", [
    ("d3q15", (65, 3, 2), 3, "zh"), ("d3q15", (130, 2, 2), 0, "random"),
    ("d2q9", (97, 5, 1), 1, "zh"), ("d2q9", (161, 3, 1), 2, "random"),
    # several tiles per row (tiled AA: x neighbours across tile edges)
    ("d3q15", (128, 3, 2), 3, "zh"), ("d2q9", (192, 4, 1), 0, "random")])
def test_rows_across_blocks(lbmc, lat, length, ct, bc, streaming):
    case = make_case(lat, length, ct, True, solids=0.1, partial=0.15 if ct % 2 else 0.0,
                     macro="random" if bc == "random" else None, micro="zh" if bc == "zh" else None,
                     seed=6)
    sm = lbmc.STREAM_AA if streaming == "aa" else lbmc.STREAM_SHIFT
    f, r = run_both(lbmc, case, 30, lbmc.F32, sm)
    assert err(f, r) <= 1e-5


def test_zero_steps_is_a_no_op(lbmc):
    case = make_case("d3q15", (9, 5, 4), seed=2)
    with lbmc.Engine.from_case(case) as eng:
        f0 = eng.f()
        eng.iterate(0, lbmc.STORE_MACROS | lbmc.REDUCE_DIAG | lbmc.SYNC)
        assert eng.step() == 0
        np.testing.assert_array_equal(eng.f(), f0)


@pytest.mark.parametrize("streaming", ["shift", "aa"])
@pytest.mark.parametrize("storage", ["f16", "f16sr"])
def test_fp16_storage_round_trips_every_finite_value(lbmc, streaming, storage):
    """Every finite FP16 bit pattern h, uploaded as f = w + h / 1024, is
    stored as exactly h and read back through the load path (one fused
    FP16 x FP16 -> FP32 FMA) as exactly h / 1024, so lbmc_fetch returns the
    uploaded f bit for bit (both sides form w + h / 1024 with one double
    rounding): subnormals and the largest values included, in the shift and
    the tiled AA layout (Lx = 64)."""
    bits = np.arange(65536, dtype=np.uint32).astype(np.uint16)
    bits = bits[(bits & 0x7C00) != 0x7C00]
    h = bits.view(np.float16).astype(np.float64)
    case = make_case("d3q15", (64, 67, 1), seed=1)
    n, q = case.n, case.q
    w = Restatement(case).equilibrium(np.ones(n), np.zeros((3, n)))[:, :1]
    dev = np.zeros(q * n)
    dev[:h.size] = h / 1024.0
    case.f0 = w + dev.reshape(q, n)
    sm = lbmc.STREAM_AA if streaming == "aa" else lbmc.STREAM_SHIFT
    with lbmc.Engine.from_case(case, init_type=lbmc.INIT_F, storage=lbmc.STORAGE_IDS[storage],
                               streaming=sm) as eng:
        got = np.asarray(eng.f()).reshape(q, n)
    np.testing.assert_array_equal(got, case.f0)
