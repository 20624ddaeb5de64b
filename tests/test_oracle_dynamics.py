"""Pins the oracle's complex128 Trotter restatement to the reference's own output.

Golden series: data_processed/probability_dynamics_n{16,20}.csv (cuStateVec
complex128 on H200; P_< printed with 7 significant digits, <d_H> with 4 decimals),
excerpted into tests/golden/series_n*.json by tests/golden/make_golden.py.
Exact propagator: oracle/ed_oracle.py restating src/connector/connector.cuh:683-805.
"""
import numpy as np
import pytest

from oracle import oracle as O
from oracle import ed_oracle

# print precision of the golden CSV (%e with 6 decimals; %.4f)
P_REL = 6e-7
DH_ABS = 5.01e-5


def _check_series(n, s, threads=0):
    bits = int(s["trap_bits"], 16)
    e0 = O.labs_energy(n, bits)
    assert e0 == s["trap_energy"]
    steps = int(round(s["t_max"] / s["dt"]))
    every = s["every"]
    p, d, nn = O.trotter_evolve(n, bits, e0, s["g"], s["dt"], steps, measure=range(0, steps + 1, every),
                                threads=threads)
    gp, gd = np.array(s["p_less"]), np.array(s["dh"])
    assert len(p) == len(gp)
    assert np.all(np.abs(p - gp) <= P_REL * np.abs(gp) + 1e-300)
    assert np.all(np.abs(d - gd) <= DH_ABS)
    assert np.all(np.abs(nn - 1.0) < 1e-10)


def test_golden_series_n16(golden):
    for s in golden("series_n16.json")["series"]:
        _check_series(16, s)


@pytest.mark.slow
def test_golden_series_n20(golden):
    for s in golden("series_n20.json")["series"]:
        _check_series(20, s)


def test_trotter_vs_exact_diagonalisation():
    # Config "plain method" shape at reduced n: the Trotter error is O(dt^2), so
    # halving dt must shrink the gap to the exact propagator about 4x.
    n, g = 8, 0.35
    e_tab = O.energy_table(n)
    starts = O.random_states(n, 42, 50)
    traps = sorted({O.steepest_descent(n, int(s))[:2] for s in starts}, key=lambda x: -x[1])
    bits, e0 = traps[0]
    times = np.arange(0, 21) * 1.0
    pe, de = ed_oracle.propagate(n, g, bits, e0, times, e_tab)
    errs = []
    for dt in (0.05, 0.025):
        steps = int(round(20.0 / dt))
        stride = int(round(1.0 / dt))
        p, d, _ = O.trotter_evolve(n, bits, e0, g, dt, steps, measure=range(0, steps + 1, stride))
        errs.append(max(np.abs(p - pe).max(), np.abs(d - de).max() / n))
    assert errs[0] < 5e-3
    assert 3.0 < errs[0] / errs[1] < 5.0


def test_sampler_schedule_and_post_processing():
    # record_trajectory: a point at every dt_trajectory from t = 0 to t_max inclusive
    cfg = dict(n=8, num_sample_points=20, shots_per_point=0, num_sampling_seeds=3, track_p_less=1,
               record_trajectory=1, seed=42, seed_stride=10007, g=0.35, dt=0.05, t_max=3.0, t_start=0.0,
               dt_sample=0.0, dt_trajectory=0.0)
    bits = O.steepest_descent(8, int(O.random_states(8, 5, 1)[0]))[0]
    r = O.sampler_run(cfg, bits)
    assert np.allclose(r["time_points"], np.arange(61) * 0.05)
    p, d, _ = O.trotter_evolve(8, bits, r["start_energy"], 0.35, 0.05, 60)
    assert np.allclose(r["p_less_history"], p, rtol=0, atol=1e-14)
    assert r["peak_p_less"] == pytest.approx(p.max())
    # delayed window: points at t_start + k * dt_sample, window average over it
    cfg.update(record_trajectory=0, t_start=1.0, dt_sample=0.5, num_sample_points=4)
    r = O.sampler_run(cfg, bits)
    assert np.allclose(r["time_points"], [1.0, 1.5, 2.0, 2.5, 3.0])
    sel = [i for i, t in enumerate(r["time_points"]) if 1.0 - 1e-9 <= t <= 2.5 + 1e-9]
    assert r["window_avg_dh"] == pytest.approx(np.mean(r["dh_history"][sel]))
    # projective sampling: shot counts per seed and totals
    cfg.update(shots_per_point=50)
    r = O.sampler_run(cfg, bits)
    assert r["total_shots_collected"] == 4 * 50
    assert [s["total_shots_collected"] for s in r["seed_stats"]] == [200, 200, 200]
    assert [s["seed"] for s in r["seed_stats"]] == [42, 42 + 10007, 42 + 2 * 10007]
    assert 0.0 <= r["success_rate"] <= 1.0
