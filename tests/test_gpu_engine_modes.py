"""The two schedules of the tile engine — the persistent dataflow kernel and one
grid launch per pass — run the same tile arithmetic and the same fixed-order
reductions, so their measured series must agree bit for bit (and the complex128
series with the oracle to 1e-10)."""
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
    e.set_option("engine_mode", 0)
    e.close()


@pytest.mark.parametrize("n,precision", [(16, bk.BK_C64), (22, bk.BK_C64), (24, bk.BK_C64), (15, bk.BK_C128),
                                         (21, bk.BK_C128), (23, bk.BK_C128)])
def test_grid_mode_equals_persistent(eng, n, precision):
    bits, e0 = bk.select_trap(n, 11, 200, 0.05)
    steps = 30
    meas = list(range(0, steps + 1, 5))
    g = np.random.default_rng(n).uniform(0.25, 0.45, steps)
    out = []
    for mode in (0, 1):
        eng.set_option("engine_mode", mode)
        out.append(eng.evolve(n, bits, g, 0.02, steps, measure=meas, e0=e0, precision=precision))
    eng.set_option("engine_mode", 0)
    for a, b in zip(out[0], out[1]):
        assert np.array_equal(a, b)


def test_grid_mode_matches_oracle_c128(eng):
    n, steps = 17, 24
    bits, e0 = bk.select_trap(n, 5, 200, 0.05)
    eng.set_option("engine_mode", 1)
    p, d, nn = eng.evolve(n, bits, 0.35, 0.05, steps, e0=e0, precision=bk.BK_C128)
    eng.set_option("engine_mode", 0)
    po, do, no = O.trotter_evolve(n, bits, e0, 0.35, 0.05, steps)
    assert np.max(np.abs(p - po)) <= 1e-10
    assert np.max(np.abs(d - do)) <= 1e-10 * n
    assert np.max(np.abs(nn - 1.0)) <= 1e-10


@pytest.mark.parametrize("w2", [4, 6])
def test_forced_split_matches_oracle_c128(eng, w2):
    """S2 width forced by the tuner's knob (the rest goes to S3): same physics."""
    n, steps = 22, 16
    bits, e0 = bk.select_trap(n, 8, 200, 0.05)
    eng.set_option("split_w2", w2)
    p, d, nn = eng.evolve(n, bits, 0.35, 0.05, steps, e0=e0, precision=bk.BK_C128)
    eng.set_option("split_w2", 0)
    po, do, _ = O.trotter_evolve(n, bits, e0, 0.35, 0.05, steps)
    assert np.max(np.abs(p - po)) <= 1e-10
    assert np.max(np.abs(d - do)) <= 1e-10 * n


def test_tuner_sweeps_and_caches(eng, tmp_path):
    from bk_b200 import tune
    path = str(tmp_path / "cache.json")
    e = tune.tune(eng, 20, bk.BK_C64, steps=4, warmup=1, cache_path=path)
    assert len(e["candidates"]) == len(tune.candidates(20, bk.BK_C64))
    assert e["amp_steps_per_s"] == max(c["amp_steps_per_s"] for c in e["candidates"])
    eng.set_option("engine_mode", 0)
    assert tune.apply(eng, 20, bk.BK_C64, cache_path=path) == e["best"]
    assert eng.get_option("engine_mode") == e["best"]["engine_mode"]
    for k in tune.KNOBS:
        eng.set_option(k, tune.DEFAULTS[k])


@pytest.mark.parametrize("n,precision", [(22, bk.BK_C64), (21, bk.BK_C128)])
def test_recomputed_energies_equal_the_table(eng, n, precision):
    """E(s) from popcounts in the pass (BK_OPT_E_SOURCE = 1) is the same integer as
    the table's: identical series in both schedules."""
    bits, e0 = bk.select_trap(n, 4, 200, 0.05)
    steps = 12
    ref = None
    for mode in (0, 1):
        for src in (0, 1):
            eng.set_option("engine_mode", mode)
            eng.set_option("e_source", src)
            out = eng.evolve(n, bits, 0.35, 0.02, steps, measure=range(0, steps + 1, 3), e0=e0, precision=precision)
            if ref is None:
                ref = out
            for a, b in zip(ref, out):
                assert np.array_equal(a, b)
    eng.set_option("engine_mode", 0)
    eng.set_option("e_source", 0)


def test_wide_a1_matches_oracle_c128(eng):
    """The 512-thread A1 of the per-pass schedule (BK_OPT_A1_WIDE): complex128
    series within 1e-10 of the oracle; complex64 within 1e-6 of the 256-thread A1
    (the same rotations in another round order)."""
    n, steps = 17, 24
    bits, e0 = bk.select_trap(n, 6, 200, 0.05)
    eng.set_option("engine_mode", 1)
    eng.set_option("a1_wide", 1)
    try:
        p, d, nn = eng.evolve(n, bits, 0.35, 0.05, steps, e0=e0, precision=bk.BK_C128)
        po, do, _ = O.trotter_evolve(n, bits, e0, 0.35, 0.05, steps)
        assert np.max(np.abs(p - po)) <= 1e-10 and np.max(np.abs(d - do)) <= 1e-10 * n
        b2, e2 = bk.select_trap(22, 6, 200, 0.05)
        pw, dw, _ = eng.evolve(22, b2, 0.35, 0.02, 40, measure=range(0, 41, 5), e0=e2, precision=bk.BK_C64)
        eng.set_option("a1_wide", 0)
        ps, ds, _ = eng.evolve(22, b2, 0.35, 0.02, 40, measure=range(0, 41, 5), e0=e2, precision=bk.BK_C64)
        assert np.max(np.abs(pw - ps)) <= C64_DP_BAR and np.max(np.abs(dw - ds)) <= C64_DH_BAR
    finally:
        eng.set_option("a1_wide", 0)
        eng.set_option("engine_mode", 0)


@pytest.mark.gpu
def test_warp_local_a1_matches_oracle(eng):
    """The warp-local A1 of the per-pass schedule (BK_OPT_A1_WIDE = 2: element
    bits 0-8 in one warp per 512-element block, the strided passes from bit 9):
    complex128 series within 1e-10 of the oracle for a one-strided-pass size
    (n = 17: S2 = 8 bits) and a two-pass size with the default and forced
    splits (n = 22: 7 + 6 by default, 4 + 9 and 9 + 4 forced);
    complex64 within 1e-6 of the 256-thread A1 at n = 24 with the table and the
    recomputed E, and at n = 28 (S2 = S3 = 9 bits); norms within 1e-5."""
    eng.set_option("engine_mode", 1)
    try:
        eng.set_option("a1_wide", 2)
        for n, w2 in ((17, 0), (22, 0), (22, 4), (22, 9)):
            bits, e0 = bk.select_trap(n, 6, 200, 0.05)
            eng.set_option("split_w2", w2)
            p, d, nn = eng.evolve(n, bits, 0.35, 0.02, 12, measure=range(0, 13, 3), e0=e0, precision=bk.BK_C128)
            po, do, no = O.trotter_evolve(n, bits, e0, 0.35, 0.02, 12, measure=list(range(0, 13, 3)))
            assert np.max(np.abs(p - po)) <= 1e-10, (n, w2)
            assert np.max(np.abs(d - do)) <= 1e-10 * n, (n, w2)
            assert np.max(np.abs(nn - no)) <= 1e-10, (n, w2)
        eng.set_option("split_w2", 0)
        for n, steps, e_source in ((24, 30, 0), (24, 30, 1), (28, 8, 0)):
            b2, e2 = bk.select_trap(n, 6, 200, 0.05)
            eng.set_option("e_source", e_source)
            out = {}
            for kernel in (0, 2):
                eng.set_option("a1_wide", kernel)
                out[kernel] = eng.evolve(n, b2, 0.35, 0.02, steps, measure=range(0, steps + 1, 2), e0=e2,
                                         precision=bk.BK_C64)
            (pw, dw, nw), (ps, ds, ns) = out[2], out[0]
            assert np.max(np.abs(pw - ps)) <= C64_DP_BAR and np.max(np.abs(dw - ds)) <= C64_DH_BAR, (n, e_source)
            # the complex64 norm itself drifts ~1e-6 over 30 steps (FP32 sums)
            assert np.max(np.abs(nw - ns)) <= 1e-5, (n, e_source)
    finally:
        eng.set_option("a1_wide", 0)
        eng.set_option("e_source", 0)
        eng.set_option("split_w2", 0)
        eng.set_option("engine_mode", 0)


@pytest.mark.gpu
def test_warp_local_a1_falls_back_above_27_element_bits(eng):
    """BK_OPT_A1_WIDE = 2 on a size whose strided passes could not take the
    remaining bits (complex64 n = 30, complex128 n = 28: more than 27 element
    bits) runs the 256-thread A1 geometry: series bit-identical to value 0."""
    eng.set_option("engine_mode", 1)
    try:
        for n, prec in ((30, bk.BK_C64), (28, bk.BK_C128)):
            bits, e0 = bk.select_trap(n, 6, 100, 0.05)
            out = {}
            for kernel in (0, 2):
                eng.set_option("a1_wide", kernel)
                out[kernel] = eng.evolve(n, bits, 0.35, 0.02, 3, measure=[0, 3], e0=e0, precision=prec)
            for a, b in zip(out[0], out[2]):
                assert np.array_equal(a, b), n
    finally:
        eng.set_option("a1_wide", 0)
        eng.set_option("engine_mode", 0)
