"""bk_b200.export: the reference connector's output files, byte for byte.

Pinned two ways (no GPU):
* the time-series CSV against rows of the reference's own
  data_processed/probability_dynamics_n{16,28}.csv (tests/golden/time_series_rows_n*.csv,
  made by tests/golden/make_golden.py): records rebuilt from the rows must print
  back to the same bytes — including `g` printed as 0.3 on the file's first row
  and 3.000000e-01 after it (the stream's float format carries over);
* all three writers against oracle/export_oracle.cpp, the writers of
  src/connector/connector.cuh:839-1155 restated on real std::ofstream objects, on
  seeded random records (several traps and g per trap, maps, empty series,
  extreme exponents, the uppercase flag the first hex trap id leaves set).
"""
import csv
import io
import json
import os
import random
import subprocess

import pytest

from bk_b200 import export as X

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
ORACLE = os.path.join(ROOT, "oracle")


def _records_from_rows(text):
    recs = []
    for row in csv.DictReader(io.StringIO(text)):
        key = (int(row["N"]), float(row["g"]), int(row["trap_rank"]), int(row["trap_energy"]), float(row["p_blind"]))
        if not recs or recs[-1][0] != key:
            recs.append((key, X.TrapRecord(n=key[0], g=key[1], trap_rank=key[2], trap_energy=key[3],
                                           p_blind=key[4])))
        r = recs[-1][1]
        r.time_points.append(float(row["time"]))
        r.p_less_history.append(float(row["p_less"]))
        r.dh_history.append(float(row["dH"]))
    return [r for _, r in recs]


@pytest.mark.parametrize("n", [16, 28])
def test_time_series_csv_matches_reference_rows(n):
    with open(os.path.join(GOLDEN, f"time_series_rows_n{n}.csv"), newline="") as f:
        text = f.read()
    recs = _records_from_rows(text)
    assert len(recs) >= 2
    assert X.time_series_csv(recs) == text
    # the carried-over format: default on the first row, scientific afterwards
    lines = text.splitlines()
    assert lines[1].split(",")[1] in ("0.3", "0.35", "0.45") and "e-01" in lines[2].split(",")[1]


@pytest.fixture(scope="module")
def oracle_bin():
    subprocess.run(["make", "-s", "-C", ORACLE, os.path.join(ORACLE, "export_oracle")], check=True,
                   capture_output=True)
    return os.path.join(ORACLE, "export_oracle")


def _tok_str(s):
    assert " " not in s and "\n" not in s
    return f"{len(s)} {s if s else '-'}"


def _tok_vec(v):
    return " ".join([str(len(v))] + [repr(float(x)) if isinstance(x, float) else str(int(x)) for x in v])


def _tok_map(m, fl):
    out = [str(len(m))]
    for k in sorted(m):
        out += [str(int(k)), repr(float(m[k])) if fl else str(int(m[k]))]
    return " ".join(out)


def _serialise(r):
    f = repr
    parts = ["R", str(r.n), f(float(r.g)), str(r.trap_rank), str(r.trap_bits), str(r.trap_energy), str(r.d_min),
             _tok_str(r.canonical_id), _tok_str(r.canonical_hex), _tok_str(r.canonical_bitstring),
             f(r.window_avg_p_less), f(r.window_avg_dh), f(r.initial_rise_rate_avg), f(r.initial_rise_rate_max),
             f(r.quantum_time_sec), _tok_vec(r.time_points), _tok_vec(r.p_less_history), _tok_vec(r.dh_history),
             f(r.p_blind), f(r.peak_p_less), f(r.peak_time), str(r.num_sampling_seeds),
             _tok_vec(r.sample_seeds), _tok_vec(r.sample_success_rates), _tok_vec(r.sample_improved_shots),
             _tok_vec(r.sample_total_shots), _tok_vec(r.sample_best_energies),
             _tok_vec(r.sample_mean_hamming_flips),
             str(r.best_d), f(r.best_d_rate), str(r.best_d_successes), str(r.best_d_trials), str(r.best_d_evals),
             _tok_map(r.rate_by_d, True), _tok_map(r.trials_by_d, False), _tok_map(r.evals_by_d, False),
             f(r.kick_time_sec), f(r.restart_rate), str(r.restart_successes), str(r.restart_trials),
             str(r.restart_evals), f(r.restart_time_sec),
             f(r.tabu_direct_rate), str(r.tabu_direct_successes), str(r.tabu_direct_trials),
             str(r.tabu_direct_evals), f(r.tabu_direct_time_sec),
             str(r.tabu_kick_d), f(r.tabu_kick_rate), str(r.tabu_kick_successes), str(r.tabu_kick_trials),
             str(r.tabu_kick_evals),
             _tok_map(r.tabu_rate_by_d, True), _tok_map(r.tabu_trials_by_d, False), _tok_map(r.tabu_evals_by_d, False),
             f(r.tabu_kick_time_sec), f(r.tabu_restart_rate), str(r.tabu_restart_successes),
             str(r.tabu_restart_trials), str(r.tabu_restart_evals), f(r.tabu_restart_time_sec), f(r.tabu_best_rate),
             _tok_str(r.tabu_best_method),
             str(r.sd_total_evaluations), str(r.tabu_total_evaluations), str(r.total_evaluations)]
    return " ".join(parts)


def _random_records(seed):
    rng = random.Random(seed)

    def val():
        k = rng.random()
        if k < 0.1:
            return 0.0
        if k < 0.15:
            return -0.0
        if k < 0.25:
            return rng.choice([1e-300, 3.5e-12, 7.25e120, 1.0, 0.5, 123456.789])
        return rng.uniform(-2, 2) * 10.0 ** rng.randint(-9, 6)

    recs = []
    for n in rng.sample([16, 20, 24, 28, 30], 3):
        for rank in rng.sample(range(1, 9), 2):
            bits = rng.getrandbits(n)
            for g in rng.sample([0.3, 0.35, 0.45, 0.1 + 0.2, 0.125, 0.345], 3):
                npt = rng.choice([0, 1, 5, 21])
                r = X.TrapRecord(n=n, g=g, trap_rank=rank, trap_bits=bits, trap_energy=rng.randint(0, 700),
                                 d_min=rng.randint(0, 9), canonical_id=rng.choice(["", f"c{rank}_{n}"]),
                                 canonical_hex=rng.choice(["", "0x" + format(bits, "X")]),
                                 canonical_bitstring=format(bits, f"0{n}b"))
                for name in ("window_avg_p_less", "window_avg_dh", "initial_rise_rate_avg", "initial_rise_rate_max",
                             "quantum_time_sec", "p_blind", "peak_p_less", "peak_time", "best_d_rate",
                             "kick_time_sec", "restart_rate", "restart_time_sec", "tabu_direct_rate",
                             "tabu_direct_time_sec", "tabu_kick_rate", "tabu_kick_time_sec", "tabu_restart_rate",
                             "tabu_restart_time_sec", "tabu_best_rate"):
                    setattr(r, name, val())
                for name in ("best_d_successes", "best_d_trials", "best_d_evals", "restart_successes",
                             "restart_trials", "restart_evals", "tabu_direct_successes", "tabu_direct_trials",
                             "tabu_direct_evals", "tabu_kick_successes", "tabu_kick_trials", "tabu_kick_evals",
                             "tabu_restart_successes", "tabu_restart_trials", "tabu_restart_evals",
                             "sd_total_evaluations", "tabu_total_evaluations", "total_evaluations"):
                    setattr(r, name, rng.randint(0, 10 ** rng.randint(1, 9)))
                r.best_d, r.tabu_kick_d = rng.randint(0, 8), rng.randint(0, 8)
                r.tabu_best_method = rng.choice(["", "direct", "kick", "restart"])
                r.time_points = [0.05 * i for i in range(npt)]
                r.p_less_history = [val() for _ in range(npt)]
                r.dh_history = [val() for _ in range(rng.choice([npt, max(npt - 2, 0)]))]
                ns = rng.choice([0, 1, 3])
                r.num_sampling_seeds = ns
                r.sample_seeds = [42 + 10007 * i for i in range(ns)]
                r.sample_success_rates = [val() for _ in range(ns)]
                r.sample_improved_shots = [rng.randint(0, 100) for _ in range(ns)]
                r.sample_total_shots = [rng.randint(0, 2000) for _ in range(ns)]
                r.sample_best_energies = [rng.randint(-5, 500) for _ in range(ns)]
                r.sample_mean_hamming_flips = [val() for _ in range(ns)]
                for m, fl in (("rate_by_d", True), ("trials_by_d", False), ("evals_by_d", False),
                              ("tabu_rate_by_d", True), ("tabu_trials_by_d", False), ("tabu_evals_by_d", False)):
                    setattr(r, m, {d: (val() if fl else rng.randint(0, 10 ** 6))
                                   for d in rng.sample(range(1, 12), rng.randint(0, 4))})
                recs.append(r)
    rng.shuffle(recs)
    return recs


@pytest.mark.parametrize("seed,n_override", [(1, 0), (2, 0), (3, 24)])
def test_writers_match_iostream_restatement(oracle_bin, tmp_path, seed, n_override):
    recs = _random_records(seed)
    rec_file = tmp_path / "records.txt"
    rec_file.write_text("\n".join(_serialise(r) for r in recs) + "\n")
    outs = [tmp_path / "results.csv", tmp_path / "ts.csv", tmp_path / "s.json"]
    subprocess.run([oracle_bin, str(rec_file)] + [str(o) for o in outs] + [str(n_override)], check=True,
                   capture_output=True)
    assert X.results_csv(recs) == outs[0].read_text()
    assert X.time_series_csv(recs) == outs[1].read_text()
    js = X.structured_json(recs, n_override)
    assert js == outs[2].read_text()
    doc = json.loads(js)  # the structured file is valid JSON
    assert doc["system"]["num_seeds"] == len({(r.n, r.trap_rank) for r in recs})
    # the uppercase flag set by the first hex trap id: later scientific numbers print with 'E'
    rows = X.results_csv(recs).splitlines()
    assert "e" in rows[1].split(",")[7] and "E" in rows[2].split(",")[7]  # window_avg_p_less, scientific


def test_write_files(tmp_path):
    r = X.TrapRecord(n=16, g=0.35, trap_rank=1, trap_bits=0xD2EE, trap_energy=24, time_points=[0.0, 0.05],
                     p_less_history=[0.0, 1e-3], dh_history=[0.0, 0.1])
    X.export_time_series_csv(str(tmp_path / "a" / "ts.csv"), [r])
    X.export_results_csv(str(tmp_path / "a" / "res.csv"), [r])
    X.export_structured_json(str(tmp_path / "a" / "s.json"), [r])
    assert (tmp_path / "a" / "ts.csv").read_text() == X.time_series_csv([r])
    assert (tmp_path / "a" / "res.csv").read_text().endswith(",0xD2EE\n")
    assert json.loads((tmp_path / "a" / "s.json").read_text())["seeds"][0]["trap_state_hex"] == "0xD2EE"


def test_window_average_and_record_mapping():
    t = [0.0, 5.0, 10.0 - 1e-10, 20.0, 38.5 + 1e-10, 40.0]
    p = [1.0, 2.0, 3.0, 4.0, 5.0, 6.0]
    # window [10, 38.5] with the connector's 1e-9 slack
    assert X.window_average(t, p, 10.0, X.window_end(10.0, 58, 0.5, 60.0)) == pytest.approx(4.0)
    assert X.window_end(10.0, 1, 0.5, 60.0) == 60.0 and X.window_end(0.0, 20, 0.0, 60.0) == 60.0
    assert X.window_average([], [], 0.0, 1.0) == 0.0
    res = {"time_points": [0.0, 1.0, 2.0], "p_less_history": [0.0, 0.5, 1.0], "dh_history": [0.0, 1.0, 2.0],
           "window_avg_dh": 1.0, "initial_rise_rate_avg": 0.5, "initial_rise_rate_max": 0.5, "d_min": 3,
           "p_blind": 0.25, "peak_p_less": 1.0, "peak_time": 2.0,
           "seed_stats": [{"seed": 42, "success_rate": 0.1, "improved_shots": 2, "total_shots_collected": 20,
                           "mean_hamming_flips": 1.5, "best_energy": 12}]}
    r = X.record_from_sampling(res, n=12, g=0.35, trap_rank=2, trap_bits=0x5A5, trap_energy=20, t_start=1.0,
                               k_sample_points=2, dt_sample=1.0, t_max=2.0, quantum_time_sec=0.25,
                               canonical_hex="0x5A5")
    assert r.d_min == 3 and r.window_avg_p_less == pytest.approx(0.75) and r.num_sampling_seeds == 1
    assert r.sample_best_energies == [12] and r.canonical_hex == "0x5A5"
    r2 = X.record_from_sampling(res, n=12, g=0.35, trap_rank=2, trap_bits=0x5A5, trap_energy=20, d_min=5)
    assert r2.d_min == 5  # a d_min already known is kept (connector.cuh:655)
    with pytest.raises(TypeError):
        X.record_from_sampling(res, n=12, g=0.35, trap_rank=2, trap_bits=1, trap_energy=20, no_such_field=1)
