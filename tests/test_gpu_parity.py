"""GPU parity of the CUDA engine against the oracle and the reference's golden data.

Tolerances (written here, per the engine's contract):
  * E(s), p_blind counts: bit-exact.
  * complex128 (fused and plain): |dP_<| <= 1e-10 and |d<d_H>| <= 1e-10 * n against the
    complex128 CPU restatement of the reference (oracle/).
  * complex64 fused: |dP_<| <= C64_DP_BAR (1e-6), |d<d_H>| <= C64_DH_BAR (1.2e-5; the
    reason is written beside the constants in tests/conftest.py).
  * golden CSVs (cuStateVec complex128, H200): print precision (7 significant digits for
    P_<, 4 decimals for <d_H>).
"""
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


def trap(n, seed):
    """A local minimum reached by steepest descent from a seeded random state."""
    start = int(O.random_states(n, seed, 1)[0])
    bits, e0, _, _ = O.steepest_descent(n, start)
    return bits, e0


def test_energy_table_bit_exact(eng):
    for n in (1, 2, 4, 8, 12, 13, 16, 20, 24, 26):
        assert np.array_equal(eng.energy_table(n), O.energy_table(n)), n


def test_p_blind_counts(eng, golden):
    for n in (12, 16, 20, 24):
        for seed in (1, 2):
            bits, e0 = trap(n, seed)
            c, p = eng.p_blind(n, e0)
            assert c == O.count_below(n, e0)
            assert p == c / float(1 << n)
    for r in golden("traps.json")["results"]["24"][::6]:
        c, p = eng.p_blind(24, int(r["trap_energy"]))
        assert p == pytest.approx(float(r["p_blind"]), rel=6e-7)


CASES = [  # n, seed, steps, dt
    (3, 1, 40, 0.05), (8, 2, 60, 0.05), (12, 3, 60, 0.05), (13, 4, 30, 0.05), (14, 5, 40, 0.05),
    (15, 6, 20, 0.05), (17, 7, 25, 0.05), (20, 8, 20, 0.02), (22, 9, 8, 0.02),
]


@pytest.mark.parametrize("n,seed,steps,dt", CASES)
def test_c128_fused_matches_oracle(eng, n, seed, steps, dt):
    bits, e0 = trap(n, seed)
    rng = np.random.default_rng(seed)
    g = rng.uniform(0.25, 0.45, size=steps)  # piecewise-constant schedule
    meas = list(range(0, steps + 1, 3)) + [steps]
    meas = sorted(set(meas))
    po, do, no = O.trotter_evolve(n, bits, e0, g, dt, steps, measure=meas)
    pg, dg, ng = eng.evolve(n, bits, g, dt, steps, measure=meas, precision=bk.BK_C128)
    assert np.max(np.abs(pg - po)) <= 1e-10
    assert np.max(np.abs(dg - do)) <= 1e-10 * n
    assert np.max(np.abs(ng - 1.0)) <= 1e-10


@pytest.mark.parametrize("n,seed,steps,dt", CASES[1:6])
def test_c128_plain_matches_oracle(eng, n, seed, steps, dt):
    bits, e0 = trap(n, seed)
    po, do, _ = O.trotter_evolve(n, bits, e0, 0.35, dt, steps)
    pg, dg, _ = eng.evolve(n, bits, 0.35, dt, steps, precision=bk.BK_C128, method=bk.BK_PLAIN)
    assert np.max(np.abs(pg - po)) <= 1e-10
    assert np.max(np.abs(dg - do)) <= 1e-10 * n


@pytest.mark.parametrize("n,seed,steps,dt", CASES)
def test_c64_fused_matches_oracle(eng, n, seed, steps, dt):
    bits, e0 = trap(n, seed)
    po, do, _ = O.trotter_evolve(n, bits, e0, 0.35, dt, steps)
    pg, dg, ng = eng.evolve(n, bits, 0.35, dt, steps, precision=bk.BK_C64)
    assert np.max(np.abs(pg - po)) <= C64_DP_BAR
    assert np.max(np.abs(dg - do)) <= C64_DH_BAR
    assert np.max(np.abs(ng - 1.0)) <= 1e-5


@pytest.mark.parametrize("n", [24, 26, 28, 30])
def test_golden_series_c128(eng, golden, n):
    for s in golden(f"series_n{n}.json")["series"]:
        bits = int(s["trap_bits"], 16)
        steps = int(round(s["t_max"] / s["dt"]))
        meas = range(0, steps + 1, s["every"])
        p, d, nn = eng.evolve(n, bits, s["g"], s["dt"], steps, measure=meas, precision=bk.BK_C128)
        gp, gd = np.array(s["p_less"]), np.array(s["dh"])
        assert np.all(np.abs(p - gp) <= 6e-7 * np.abs(gp) + 1e-300), (n, s["g"])
        assert np.all(np.abs(d - gd) <= 5.01e-5), (n, s["g"])
        assert np.max(np.abs(nn - 1.0)) < 1e-9


def test_c64_vs_c128_n24_config(eng):
    # N = 24 trap, g = 0.35, dt = 0.02, 1000 steps, measured every 10 steps
    bits, e0 = 0xFAD33, 56
    meas = range(0, 1001, 10)
    p64, d64, n64 = eng.evolve(24, bits, 0.35, 0.02, 1000, measure=meas, precision=bk.BK_C64)
    p128, d128, _ = eng.evolve(24, bits, 0.35, 0.02, 1000, measure=meas, precision=bk.BK_C128)
    assert np.max(np.abs(p64 - p128)) <= C64_DP_BAR
    assert np.max(np.abs(d64 - d128)) <= C64_DH_BAR
    assert np.max(np.abs(n64 - 1.0)) <= 1e-4


def test_strang_ordering_same_probabilities(eng):
    n, steps = 14, 30
    bits, e0 = trap(n, 11)
    pr, dr, _ = eng.evolve(n, bits, 0.35, 0.05, steps, precision=bk.BK_C128)
    sr = eng.export_state(n)
    ps, ds, _ = eng.evolve(n, bits, 0.35, 0.05, steps, precision=bk.BK_C128, ordering=bk.BK_ORDER_STRANG)
    ss = eng.export_state(n)
    assert np.allclose(pr, ps, atol=1e-14) and np.allclose(dr, ds, atol=1e-13)
    assert np.allclose(np.abs(sr) ** 2, np.abs(ss) ** 2, atol=1e-14)
    _, _, _, so = O.trotter_evolve(n, bits, e0, 0.35, 0.05, steps, measure=[steps], want_state=True)
    assert np.max(np.abs(sr - so)) <= 1e-10


def test_sampling_matches_inverse_cdf(eng):
    n, steps = 10, 40
    bits, e0 = trap(n, 12)
    eng.evolve(n, bits, 0.35, 0.05, steps, measure=[steps], precision=bk.BK_C128)
    st = eng.export_state(n)
    r = O.uniform_randoms(42, 20000)
    got = eng.sample(r)
    ref = O.sample_indices(n, st, r)
    assert np.mean(got == ref) >= 0.999
    # chi^2 against |psi|^2 on the complex64 path
    eng.evolve(n, bits, 0.35, 0.05, steps, measure=[steps], precision=bk.BK_C64)
    r = O.uniform_randoms(7, 200000)
    counts = np.bincount(eng.sample(r).astype(np.int64), minlength=1 << n)
    prob = np.abs(st) ** 2
    keep = prob * len(r) > 5
    chi2 = np.sum((counts[keep] - prob[keep] * len(r)) ** 2 / (prob[keep] * len(r)))
    dof = int(keep.sum()) - 1
    assert chi2 < dof + 6 * np.sqrt(2 * dof)


def test_host_side_errors(eng):
    with pytest.raises(bk.BkError) as e:
        eng.evolve(31, 0, 0.35, 0.05, 2)
    assert e.value.status == bk._lib.BK_ERR_UNSUPPORTED
    with pytest.raises(bk.BkError) as e:
        eng.evolve(10, 0, float("nan"), 0.05, 2)
    assert e.value.status == bk._lib.BK_ERR_INVALID
    with pytest.raises(bk.BkError) as e:
        eng.evolve(10, 0, 0.35, 0.05, -1)
    assert e.value.status == bk._lib.BK_ERR_INVALID
    # the context stays usable after rejected calls
    p, _, _ = eng.evolve(10, 0, 0.35, 0.05, 2)
    assert len(p) == 3


def test_c64_state_infidelity_n24_config(eng):
    """complex64 against complex128 at the N = 24 configuration (1000 steps):
    state infidelity 1 - |<psi_64|psi_128>|^2 of the exported statevectors."""
    bits = 0xFAD33
    eng.evolve(24, bits, 0.35, 0.02, 1000, measure=[1000], precision=bk.BK_C64)
    s64 = eng.export_state(24)
    eng.evolve(24, bits, 0.35, 0.02, 1000, measure=[1000], precision=bk.BK_C128)
    s128 = eng.export_state(24)
    ov = np.vdot(s64, s128) / (np.linalg.norm(s64) * np.linalg.norm(s128))
    infidelity = 1.0 - abs(ov) ** 2
    assert infidelity <= 1e-8, infidelity


def test_plain_config_n12_against_oracle_and_ed(eng):
    """The N = 12 configuration: complex128, dt = 0.05, 400 steps (T = 20), P_< and
    <d_H> every 10 steps; equal to the oracle to 1e-10 and to dense exact
    diagonalisation (4096 x 4096) within the O(dt^2) Trotter error."""
    from oracle import ed_oracle
    n, dt, steps = 12, 0.05, 400
    bits, e0 = bk.select_trap(n, 42, 1000, 0.05)
    meas = range(0, steps + 1, 10)
    p, d, nn = eng.evolve(n, bits, 0.35, dt, steps, measure=meas, e0=e0, precision=bk.BK_C128)
    po, do, _ = O.trotter_evolve(n, bits, e0, 0.35, dt, steps, measure=meas)
    assert np.max(np.abs(p - po)) <= 1e-10 and np.max(np.abs(d - do)) <= 1e-10 * n
    pe, de = ed_oracle.propagate(n, 0.35, bits, e0, np.arange(0, steps + 1, 10) * dt, O.energy_table(n))
    assert np.max(np.abs(p - pe)) <= 5e-3
    assert np.max(np.abs(d - de)) <= 5e-3 * n
