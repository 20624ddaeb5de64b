"""Adjoint gradient (bk_adjoint) on the GPU.

Pinned three ways: per-step gradients against the complex128 adjoint oracle
(itself pinned to finite differences on the CPU) for every pass geometry of the
tile engine; segment gradients against central finite differences (h = 1e-5)
of the engine's own complex128 forward run on the N = 22, 64-segment,
1280-step schedule; and the objective against bk_evolve's final measurement.
Tolerances: complex128 1e-9 relative to the largest gradient; complex64 the
float error of 1280 rounded steps, stated per test."""
import numpy as np
import pytest

import bk_b200 as bk
from bk_b200.adjoint import TrotterSchedule, optimize
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def eng():
    e = bk.Engine(0)
    yield e
    e.close()


def _case(n, nseg, T, seed):
    rng = np.random.default_rng(seed)
    bits, e0 = bk.select_trap(n, 42 + seed, 200, 0.05)
    gs = rng.uniform(0.25, 0.45, nseg)
    return bits, e0, gs, O.segment_steps(T, nseg)


# n covers the pass geometries: S2 width <= 4, 5..8, 9 (lane-shuffle bit), and S2 + S3
@pytest.mark.parametrize("n,T,K", [(13, 48, 16), (16, 48, 16), (18, 40, 16), (21, 24, 8), (22, 24, 8)])
def test_adjoint_c128_matches_oracle(eng, n, T, K):
    bits, e0, gs, seg = _case(n, 6 if T % 6 == 0 else 4, T, n)
    val, grad, st = eng.adjoint(n, bits, gs, 0.05, T, e0=e0, precision=bk.BK_C128, checkpoint_every=K,
                                per_step=True)
    oval, ograd = O.trotter_adjoint(n, bits, e0, gs[seg], 0.05, T)
    scale = np.max(np.abs(ograd))
    assert scale > 0
    assert abs(val - oval) <= 1e-10
    assert np.max(np.abs(st["grad_steps"] - ograd)) <= 1e-9 * scale
    assert np.max(np.abs(grad - np.bincount(seg, weights=ograd))) <= 1e-9 * scale * T
    assert st["n_checkpoints"] == (T - 1) // K
    assert st["max_drift"] <= 1e-11


@pytest.mark.parametrize("n", [14, 18, 20, 22, 23])
def test_adjoint_c64_matches_oracle(eng, n):
    T, K = (24, 8) if n >= 22 else (40, 16)
    bits, e0, gs, seg = _case(n, 4, T, n)
    val, grad, st = eng.adjoint(n, bits, gs, 0.05, T, e0=e0, precision=bk.BK_C64, checkpoint_every=K,
                                per_step=True)
    oval, ograd = O.trotter_adjoint(n, bits, e0, gs[seg], 0.05, T)
    scale = np.max(np.abs(ograd))
    assert abs(val - oval) <= 1e-6
    # complex64 state (FP32 butterflies), FP32 cross terms per round, FP64 above
    assert np.max(np.abs(st["grad_steps"] - ograd)) <= 1e-4 * scale
    assert st["max_drift"] <= 1e-4


@pytest.mark.parametrize("n,adj_a1", [(18, 0), (22, 0), (23, 0), (22, 1)])
def test_adjoint_c64_phase_table_matches_oracle(eng, n, adj_a1):
    """The reverse A1 pass with the full complex64 phase table (BK_OPT_PHASE_TABLE:
    D^dagger as the negated half-angle shear rotations of each level's entry), in
    the 12-bit and the warp-local layouts: the same bars as the level-table path."""
    T, K = (24, 8) if n >= 22 else (40, 16)
    bits, e0, gs, seg = _case(n, 4, T, n)
    eng.set_option("phase_table", 1)
    eng.set_option("adj_a1", adj_a1)
    try:
        val, grad, st = eng.adjoint(n, bits, gs, 0.05, T, e0=e0, precision=bk.BK_C64, checkpoint_every=K,
                                    per_step=True)
    finally:
        eng.set_option("phase_table", 0)
        eng.set_option("adj_a1", 0)
    oval, ograd = O.trotter_adjoint(n, bits, e0, gs[seg], 0.05, T)
    scale = np.max(np.abs(ograd))
    assert abs(val - oval) <= 1e-6
    assert np.max(np.abs(st["grad_steps"] - ograd)) <= 1e-4 * scale
    assert st["max_drift"] <= 1e-4


def test_adjoint_d_h_objective_c128(eng):
    n, T = 16, 36
    bits, e0, gs, seg = _case(n, 6, T, 5)
    val, grad, st = eng.adjoint(n, bits, gs, 0.05, T, e0=e0, precision=bk.BK_C128, objective=bk.BK_OBJ_D_H,
                                checkpoint_every=10, per_step=True)
    oval, ograd = O.trotter_adjoint(n, bits, e0, gs[seg], 0.05, T, objective=1)
    assert abs(val - oval) <= 1e-10 * n
    assert np.max(np.abs(st["grad_steps"] - ograd)) <= 1e-9 * np.max(np.abs(ograd))


@pytest.mark.parametrize("precision", [bk.BK_C64, bk.BK_C128])
def test_adjoint_value_is_the_forward_measurement(eng, precision):
    n, T = 20, 60
    bits, e0, gs, seg = _case(n, 5, T, 9)
    val, _, st = eng.adjoint(n, bits, gs, 0.02, T, e0=e0, precision=precision, checkpoint_every=16)
    p, d, nn = eng.evolve(n, bits, gs[seg], 0.02, T, measure=[T], e0=e0, precision=precision)
    assert st["norm"] == nn[0]
    if precision == bk.BK_C128:
        assert val == p[0]
    else:
        # bk_evolve returns complex64 sums divided by the norm; the adjoint's
        # objective is the raw sum whose gradient it returns
        assert val == pytest.approx(p[0] * nn[0], rel=1e-14, abs=0.0)


def test_adjoint_segment_gradients_match_finite_differences_n22(eng):
    """N = 22, 64 segments, 1280 steps (20 per segment), checkpoints every 128;
    central differences h = 1e-5 of the complex128 forward run."""
    n, nseg, T, dt, h = 22, 64, 1280, 0.02, 1e-5
    bits, e0 = bk.select_trap(n, 42, 1000, 0.05)
    gs = np.random.default_rng(42).uniform(0.25, 0.45, nseg)
    seg = O.segment_steps(T, nseg)
    fd = np.zeros(nseg)
    for j in range(nseg):
        v = []
        for sgn in (1.0, -1.0):
            gg = gs.copy()
            gg[j] += sgn * h
            v.append(eng.evolve(n, bits, gg[seg], dt, T, measure=[T], e0=e0, precision=bk.BK_C128)[0][0])
        fd[j] = (v[0] - v[1]) / (2 * h)
    scale = np.max(np.abs(fd))
    _, g128, st128 = eng.adjoint(n, bits, gs, dt, T, e0=e0, precision=bk.BK_C128, checkpoint_every=128)
    _, g64, st64 = eng.adjoint(n, bits, gs, dt, T, e0=e0, precision=bk.BK_C64, checkpoint_every=128)
    assert st128["n_checkpoints"] == 9
    assert np.max(np.abs(g128 - fd)) <= 1e-7 * scale + 1e-10
    assert np.max(np.abs(g64 - fd)) <= 1e-3 * scale


def test_adam_on_the_schedule_raises_p_less(eng):
    n, nseg, T = 16, 8, 160
    bits, e0 = bk.select_trap(n, 3, 200, 0.05)
    g0 = np.random.default_rng(1).uniform(0.25, 0.45, nseg)
    sched = TrotterSchedule(eng, n, bits, g0, 0.05, T, precision=bk.BK_C128, checkpoint_every=32, e0=e0)
    hist = optimize(sched, steps=20, lr=0.02)
    assert len(hist) == 21
    assert hist[-1] > hist[0]


def test_adjoint_rejects_bad_input(eng):
    with pytest.raises(bk.BkError) as e:
        eng.adjoint(12, 5, [0.3], 0.05, 10, precision=bk.BK_C64)
    assert e.value.status == bk._lib.BK_ERR_UNSUPPORTED
    with pytest.raises(bk.BkError) as e:
        eng.adjoint(16, 5, [0.3, 0.4], 0.05, 9, precision=bk.BK_C64)
    assert e.value.status == bk._lib.BK_ERR_INVALID
    with pytest.raises(bk.BkError) as e:
        eng.adjoint(16, 5, [0.3, 0.4], 0.05, 4, segment_of_step=[0, 1, 2, 0], precision=bk.BK_C64)
    assert e.value.status == bk._lib.BK_ERR_INVALID


def test_adjoint_n28_complex64_against_complex128(eng):
    """The large configuration's adjoint: N = 28 (three-pass dual sweep, S2 + S3),
    checkpoints every 16 steps; complex64 gradients within 1e-3 of complex128."""
    n, T, nseg = 28, 64, 4
    bits, e0 = bk.select_trap(n, 42, 200, 0.01)
    gs = np.random.default_rng(28).uniform(0.25, 0.45, nseg)
    v64, g64, st64 = eng.adjoint(n, bits, gs, 0.02, T, e0=e0, precision=bk.BK_C64, checkpoint_every=16)
    v128, g128, st128 = eng.adjoint(n, bits, gs, 0.02, T, e0=e0, precision=bk.BK_C128, checkpoint_every=16)
    assert st64["n_checkpoints"] == 3 and st128["max_drift"] <= 1e-11 and st64["max_drift"] <= 1e-4
    assert abs(v64 - v128) <= 1e-6
    assert np.max(np.abs(g64 - g128)) <= 1e-3 * np.max(np.abs(g128))


# warp-local reverse A1 (BK_OPT_ADJ_A1 = 1): element bits 0-8 per warp, strided
# passes from bit 9 — one S2 of 4 bits (n = 13), of 9 bits with the lane-shuffle
# bit (n = 18), S2 + S3 (n = 22: 7 + 6)
@pytest.mark.parametrize("n,T,K", [(13, 48, 16), (18, 40, 16), (22, 24, 8)])
def test_adjoint_warp_local_a1_c128_matches_oracle(eng, n, T, K):
    bits, e0, gs, seg = _case(n, 6 if T % 6 == 0 else 4, T, n)
    prev = eng.get_option("adj_a1")
    eng.set_option("adj_a1", 1)
    try:
        val, grad, st = eng.adjoint(n, bits, gs, 0.05, T, e0=e0, precision=bk.BK_C128, checkpoint_every=K,
                                    per_step=True)
    finally:
        eng.set_option("adj_a1", prev)
    oval, ograd = O.trotter_adjoint(n, bits, e0, gs[seg], 0.05, T)
    scale = np.max(np.abs(ograd))
    assert abs(val - oval) <= 1e-10
    assert np.max(np.abs(st["grad_steps"] - ograd)) <= 1e-9 * scale
    assert st["max_drift"] <= 1e-11


@pytest.mark.parametrize("n", [14, 23])
def test_adjoint_warp_local_a1_c64_matches_oracle(eng, n):
    T, K = (24, 8) if n >= 22 else (40, 16)
    bits, e0, gs, seg = _case(n, 4, T, n)
    prev = eng.get_option("adj_a1")
    eng.set_option("adj_a1", 1)
    try:
        val, grad, st = eng.adjoint(n, bits, gs, 0.05, T, e0=e0, precision=bk.BK_C64, checkpoint_every=K,
                                    per_step=True)
    finally:
        eng.set_option("adj_a1", prev)
    oval, ograd = O.trotter_adjoint(n, bits, e0, gs[seg], 0.05, T)
    assert abs(val - oval) <= 1e-6
    assert np.max(np.abs(st["grad_steps"] - ograd)) <= 1e-4 * np.max(np.abs(ograd))
    assert st["max_drift"] <= 1e-4


def test_adjoint_n28_full_schedule_checkpoints_sized_to_memory(eng):
    """The large configuration's adjoint run in full: N = 28, 2000 steps (40
    segments of 50, g_j ~ U[0.25, 0.45]), dt = 0.02, checkpoint interval left to
    bk_adjoint's free-memory rule (128 steps, enlarged only when the checkpoints
    would not fit in free HBM). complex64 against complex128 over the whole
    run: objective within 1e-6, gradients within 1e-3 of the largest; the
    objective equals bk_evolve's P_<(T) of the same schedule."""
    n, T, nseg = 28, 2000, 40
    bits, e0 = bk.select_trap(n, 42, 4000, 0.01)
    gs = np.random.default_rng(2028).uniform(0.25, 0.45, nseg)
    seg = O.segment_steps(T, nseg)
    v64, g64, st64 = eng.adjoint(n, bits, gs, 0.02, T, e0=e0, precision=bk.BK_C64, checkpoint_every=0)
    v128, g128, st128 = eng.adjoint(n, bits, gs, 0.02, T, e0=e0, precision=bk.BK_C128, checkpoint_every=0)
    for st in (st64, st128):
        assert st["checkpoint_every"] >= 128
        assert st["n_checkpoints"] == (T - 1) // st["checkpoint_every"]
    assert st64["max_drift"] <= 1e-4 and st128["max_drift"] <= 1e-11
    assert abs(v64 - v128) <= 1e-6
    assert np.max(np.abs(g64 - g128)) <= 1e-3 * np.max(np.abs(g128))
    p, _, _ = eng.evolve(n, bits, gs[seg], 0.02, T, measure=[T], e0=e0, precision=bk.BK_C128)
    assert abs(v128 - p[-1]) <= 1e-10
