"""GPU parity of the reference's ISampler::sample() (src/sampling/sampler.cuh:412-707)
run through the C ABI (bk_sampler_run) against the oracle's restatement of the same
semantics (oracle/trotter_oracle.cpp, orc_sampler_run) and the golden results CSVs.

Tolerances: trajectories 1e-10 (complex128); integer fields exact; shot statistics
exact when every draw matches the oracle's inverse CDF (checked), else within the
observed mismatch fraction."""
import numpy as np
import pytest

import bk_b200 as bk
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def eng():
    e = bk.Engine(0)
    yield e
    e.close()


def _oracle_cfg(n, **kw):
    cfg = dict(n=n, num_sample_points=20, shots_per_point=100, num_sampling_seeds=3, track_p_less=1,
               record_trajectory=0, seed=42, seed_stride=10007, g=0.5, dt=0.05, t_max=60.0, t_start=0.0,
               dt_sample=0.0, dt_trajectory=0.0)
    cfg.update({k: (int(v) if isinstance(v, bool) else v) for k, v in kw.items()})
    return cfg


@pytest.mark.parametrize("kw", [
    dict(record_trajectory=True, shots_per_point=0, t_max=3.0, g=0.35),
    dict(track_p_less=True, shots_per_point=0, t_max=4.0, t_start=1.0, dt_sample=0.25, num_sample_points=8),
    dict(track_p_less=True, shots_per_point=64, t_max=2.0, t_start=0.5, dt_sample=0.5, num_sample_points=3),
    dict(track_p_less=True, shots_per_point=32, t_max=1.0, num_sample_points=4, num_sampling_seeds=2),
])
def test_sampler_matches_oracle(eng, kw):
    n = 10
    bits = O.steepest_descent(n, int(O.random_states(n, 9, 1)[0]))[0]
    got = eng.sampler_run(bits, n=n, verbose=False, **kw)
    ref = O.sampler_run(_oracle_cfg(n, **kw), bits)
    assert got["start_energy"] == ref["start_energy"]
    assert got["d_min"] == ref["d_min"]
    assert got["p_blind"] == ref["p_blind"]
    assert np.array_equal(got["time_points"], ref["time_points"])
    assert np.max(np.abs(got["p_less_history"] - ref["p_less_history"]), initial=0) <= 1e-10
    assert np.max(np.abs(got["dh_history"] - ref["dh_history"]), initial=0) <= 1e-10 * n
    assert got["peak_time"] == ref["peak_time"]
    for k in ("peak_p_less", "window_avg_dh", "initial_rise_rate_avg", "initial_rise_rate_max"):
        assert got[k] == pytest.approx(ref[k], abs=1e-9), k
    assert got["total_shots_collected"] == ref["total_shots_collected"]
    assert [s["seed"] for s in got["seed_stats"]] == [s["seed"] for s in ref["seed_stats"]]
    assert [s["total_shots_collected"] for s in got["seed_stats"]] == \
        [s["total_shots_collected"] for s in ref["seed_stats"]]
    if kw.get("shots_per_point", 100) > 0:
        # draws agree unless a uniform falls within rounding of a CDF boundary
        assert abs(got["improved_shots"] - ref["improved_shots"]) <= 2
        assert got["unique_basis_size"] == pytest.approx(ref["unique_basis_size"], abs=3)


def test_sampler_golden_n16(eng, golden):
    # trajectory of the reference's own run: N=16 trap 0x7CCA, g=0.35, dt=0.05, t_max=60
    s = [x for x in golden("series_n16.json")["series"] if x["trap_rank"] == 8 and abs(x["g"] - 0.35) < 1e-12][0]
    # the connector's QuantumConfig defaults (src/config/config.hpp:102-116): window [10, 38.5]
    r = eng.sampler_run(int(s["trap_bits"], 16), n=16, g=0.35, dt=0.05, t_max=60.0, record_trajectory=True,
                        shots_per_point=0, t_start=10.0, dt_sample=1.5, num_sample_points=20, verbose=False)
    gp = np.array(s["p_less"])
    assert np.all(np.abs(r["p_less_history"] - gp) <= 6e-7 * np.abs(gp) + 1e-300)
    assert np.all(np.abs(r["dh_history"] - np.array(s["dh"])) <= 5.01e-5)
    row = [x for x in golden("traps.json")["results"]["16"] if x["trap_bits"] == s["trap_bits"]
           and abs(float(x["g"]) - 0.35) < 1e-12][0]
    assert r["d_min"] == int(row["d_min"])
    assert r["p_blind"] == pytest.approx(float(row["p_blind"]), rel=6e-7)
    assert r["peak_p_less"] == pytest.approx(float(row["peak_p_less"]), rel=6e-7)
    assert r["peak_time"] == pytest.approx(float(row["peak_time"]))
    assert r["window_avg_dh"] == pytest.approx(float(row["window_avg_dh"]), abs=5.01e-5)


def test_sampler_rejects_large_n(eng):
    with pytest.raises(bk.BkError) as e:
        eng.sampler_run(0, n=32, verbose=False)
    assert e.value.status == bk._lib.BK_ERR_UNSUPPORTED


def test_d_min_matches_oracle(eng, golden):
    for n in (10, 16, 20, 24):
        for seed in (1, 2, 3):
            bits = O.steepest_descent(n, int(O.random_states(n, seed, 1)[0]))[0]
            e = O.labs_energy(n, bits)
            assert eng.d_min(n, bits, e) == O.d_min(n, bits, e)
            assert eng.d_min(n, bits, e, 2) == O.d_min(n, bits, e, 2)
    for n_s in ("26", "28", "30"):
        for r in golden("traps.json")["results"][n_s][::3]:
            assert eng.d_min(int(n_s), int(r["trap_bits"], 16), int(r["trap_energy"])) == int(r["d_min"])


def test_sampling_segments_do_not_disturb_the_evolution(eng):
    # complex64 n = 16 runs on the persistent engine, split into launches at the
    # sampling points; the measured series must equal the unsampled run exactly
    n = 16
    bits = O.steepest_descent(n, int(O.random_states(n, 4, 1)[0]))[0]
    common = dict(n=n, g=0.35, dt=0.05, t_max=2.0, track_p_less=True, verbose=False, precision=bk.BK_C64)
    a = eng.sampler_run(bits, shots_per_point=0, t_start=0.0, dt_sample=0.05, num_sample_points=41, **common)
    b = eng.sampler_run(bits, shots_per_point=64, t_start=0.5, dt_sample=0.25, num_sample_points=5, **common)
    tb = np.round(b["time_points"] / 0.05).astype(int)
    assert np.array_equal(a["p_less_history"][tb], b["p_less_history"])
    assert b["total_shots_collected"] == 5 * 64


def test_sampling_c64_planar_vs_c128(eng):
    n = 16
    bits = O.steepest_descent(n, int(O.random_states(n, 6, 1)[0]))[0]
    kw = dict(n=n, g=0.35, dt=0.05, t_max=3.0, shots_per_point=200, t_start=1.0, dt_sample=0.5,
              num_sample_points=5, num_sampling_seeds=2, verbose=False)
    r64 = eng.sampler_run(bits, precision=bk.BK_C64, **kw)
    r128 = eng.sampler_run(bits, precision=bk.BK_C128, **kw)
    assert np.array_equal(r64["time_points"], r128["time_points"])
    assert np.max(np.abs(r64["p_less_history"] - r128["p_less_history"])) <= 1e-6
    # same uniforms, CDFs within complex64 rounding: nearly every draw identical
    assert abs(r64["improved_shots"] - r128["improved_shots"]) <= 3
    assert [s["total_shots_collected"] for s in r64["seed_stats"]] == [s["total_shots_collected"] for s in r128["seed_stats"]]
