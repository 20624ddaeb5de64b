"""Engine mode 2: the A1 pass as a grid launch and both strided passes as ONE
persistent launch: the high-bit pass (S3) first, then the middle-bit pass (S2)
re-reading from L2 the slabs S3 has just written. The Rx gates of different
qubits commute, so this is the same step as one launch per pass (mode 1, S2
then S3) up to the rounding of the other order: complex128 agrees with mode 1 to
1e-12 and with the oracle to 1e-10 (the reference's step,
src/sampling/sampler.cuh:604-618), complex64 within its parity bars; the slab lag
only changes the schedule, so results are bit-identical across lags."""
import numpy as np
import pytest

import bk_b200 as bk
from conftest import C64_DH_BAR, C64_DP_BAR
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def eng():
    e = bk.Engine(0)
    yield e
    e.close()


def _run(eng, n, precision, mode, a1, w2, lag=3, steps=12):
    bits, e0 = bk.select_trap(n, 13, 200, 0.05)
    g = np.random.default_rng(n).uniform(0.25, 0.45, steps)
    eng.set_option("engine_mode", mode)
    eng.set_option("a1_wide", a1)
    eng.set_option("split_w2", w2)
    eng.set_option("slab_lag", lag)
    try:
        return eng.evolve(n, bits, g, 0.02, steps, measure=range(0, steps + 1, 3), e0=e0, precision=precision), \
            (bits, e0, g)
    finally:
        eng.set_option("engine_mode", 0)
        eng.set_option("a1_wide", 0)
        eng.set_option("split_w2", 0)
        eng.set_option("slab_lag", 3)


# n, precision, A1 kernel (0: 256 threads, 1: 512 threads, 2: warp-local), S2 width (0: default)
CASES = [
    (22, bk.BK_C64, 0, 4), (24, bk.BK_C64, 0, 0), (24, bk.BK_C64, 1, 5), (26, bk.BK_C64, 1, 7),
    (24, bk.BK_C64, 2, 0), (26, bk.BK_C64, 2, 8), (28, bk.BK_C64, 1, 7), (28, bk.BK_C64, 2, 0),
    (21, bk.BK_C128, 0, 4), (23, bk.BK_C128, 1, 0), (25, bk.BK_C128, 2, 0),
    (16, bk.BK_C64, 0, 0),  # a single strided pass: mode 2 runs it as mode 1
]


@pytest.mark.parametrize("n,precision,a1,w2", CASES)
def test_fused_strided_matches_per_pass(eng, n, precision, a1, w2):
    steps = 12 if n < 28 else 6
    (pf, df, nf), _ = _run(eng, n, precision, 2, a1, w2, steps=steps)
    (pp, dp, np_), _ = _run(eng, n, precision, 1, a1, w2, steps=steps)
    if precision == bk.BK_C128:
        assert np.max(np.abs(pf - pp)) <= 1e-12 and np.max(np.abs(df - dp)) <= 1e-12 * n
        assert np.max(np.abs(nf - np_)) <= 1e-12
    else:
        assert np.max(np.abs(pf - pp)) <= C64_DP_BAR and np.max(np.abs(df - dp)) <= C64_DH_BAR
        assert np.max(np.abs(nf - np_)) <= 1e-5


@pytest.mark.parametrize("lag", [1, 2, 8])
def test_slab_lag_does_not_change_results(eng, lag):
    ref, _ = _run(eng, 24, bk.BK_C64, 2, 1, 5, lag=3)
    got, _ = _run(eng, 24, bk.BK_C64, 2, 1, 5, lag=lag)
    for a, b in zip(ref, got):
        assert np.array_equal(a, b)


def test_fused_strided_matches_oracle_c128(eng):
    n, steps = 21, 12
    (p, d, nn), (bits, e0, g) = _run(eng, n, bk.BK_C128, 2, 0, 4, steps=steps)
    po, do, _ = O.trotter_evolve(n, bits, e0, g, 0.02, steps, measure=range(0, steps + 1, 3))
    assert np.max(np.abs(p - po)) <= 1e-10
    assert np.max(np.abs(d - do)) <= 1e-10 * n
    assert np.max(np.abs(nn - 1.0)) <= 1e-10


def test_fused_strided_timeout_leaves_context_usable(eng):
    """A bounded wait of the fused launch that runs out (the persistent engine's
    hook does not reach mode 2, so the wait bound itself is made tiny while a
    slab dependency is still open) must come back as an error or as a correct
    result, never as a hang, and the context must keep working."""
    n = 24
    bits, e0 = bk.select_trap(n, 13, 200, 0.05)
    eng.set_option("engine_mode", 2)
    eng.set_option("wait_polls", 1000)
    try:
        try:
            eng.evolve(n, bits, 0.35, 0.02, 4, measure=[4], e0=e0, precision=bk.BK_C64)
        except bk.BkError as e:
            assert e.status == bk._lib.BK_ERR_TIMEOUT
    finally:
        eng.set_option("wait_polls", 0)
        eng.set_option("engine_mode", 0)
    p, d, _ = eng.evolve(n, bits, 0.35, 0.02, 4, measure=[4], e0=e0, precision=bk.BK_C64)
    eng.set_option("engine_mode", 2)
    try:
        p2, d2, _ = eng.evolve(n, bits, 0.35, 0.02, 4, measure=[4], e0=e0, precision=bk.BK_C64)
    finally:
        eng.set_option("engine_mode", 0)
    assert abs(p2[0] - p[0]) <= C64_DP_BAR and abs(d2[0] - d[0]) <= C64_DH_BAR


@pytest.mark.parametrize("n,precision,mode", [(24, bk.BK_C64, 1), (28, bk.BK_C64, 2), (23, bk.BK_C128, 2)])
def test_half_tile_warp_local_a1_equals_full_tile(eng, n, precision, mode):
    """BK_OPT_A1_WIDE = 3 runs the warp-local A1 with 4-warp CTAs over 32 KB half
    tiles: every element gets the same arithmetic as with value 2, so the state
    is bit-identical; the measurements sum twice as many per-tile partials, in
    another fixed order, so they agree to FP64 rounding."""
    steps = 12 if n < 28 else 6
    out = {}
    for a1 in (2, 3):
        out[a1], _ = _run(eng, n, precision, mode, a1, 0, steps=steps)
        out[a1] = out[a1] + (eng.export_state(n),)
    (p2, d2, n2, s2), (p3, d3, n3, s3) = out[2], out[3]
    assert np.array_equal(s2, s3)
    assert np.max(np.abs(p2 - p3)) <= 1e-14 and np.max(np.abs(d2 - d3)) <= 1e-13 * n
    assert np.max(np.abs(n2 - n3)) <= 1e-14


@pytest.mark.parametrize("n,precision", [(18, bk.BK_C64), (24, bk.BK_C64), (27, bk.BK_C64), (22, bk.BK_C128)])
@pytest.mark.parametrize("lag", [1, 2])
def test_self_served_groups_equal_producer_schedule(eng, n, precision, lag):
    """Engine mode 3 (two compute groups claiming and loading their own tiles,
    no producer warp) runs the same tiles in the same per-slab order as mode 2:
    identical series and state."""
    bits, e0 = bk.select_trap(n, 42, 300, 0.05)
    meas = list(range(0, 25, 4))
    out = {}
    try:
        for mode in (2, 3):
            eng.set_option("engine_mode", mode)
            eng.set_option("slab_lag", lag)
            out[mode] = eng.evolve(n, bits, 0.35, 0.02, 24, measure=meas, e0=e0, precision=precision) + \
                (eng.export_state(n),)
    finally:
        eng.set_option("engine_mode", 0)
        eng.set_option("slab_lag", 3)
    for a, b in zip(out[2], out[3]):
        assert np.array_equal(a, b), (n, lag)
