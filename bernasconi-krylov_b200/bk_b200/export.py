"""Benchmark output files in the reference connector's formats.

The reference connector writes three files per run (src/connector/connector.cuh):
the time-series CSV (`export_time_series_csv`, :906-932), the results CSV
(`export_results_csv`, :839-904) and the structured JSON
(`export_structured_json`, :934-1155); its scripts (`compute_d_min.py`,
`plot_probability_dynamics.py`, `plot_paper_figures.py`) read them. This module
writes the same bytes from this engine's results, so those scripts run
unchanged. The reference writes through one `std::ofstream` whose float format
(default / fixed / scientific, precision) and `uppercase` flag carry over from
one field to the next — e.g. after the first row, `g` prints in the scientific
form left by the previous row's `p_blind`, and after the first hex trap id every
scientific number prints with `E` — and `_Stream` reproduces that state machine.

`TrapRecord` mirrors the connector's `SingleTrapBenchmark` (:26-118) with its
defaults; `record_from_sampling` fills the quantum fields from
`Engine.sampler_run` the way `run_quantum_simulation` (:619-829) does, including
the window-averaged P_< over [t_start, avg_end] (:817-829). The classical
baseline fields (kick, restart and tabu searches) are outside this engine and
keep their defaults unless the caller fills them.
"""
import math
import os
from dataclasses import dataclass, field
from typing import Dict, List


@dataclass
class TrapRecord:
    n: int = 0
    g: float = 0.0
    trap_rank: int = 0
    trap_bits: int = 0
    trap_energy: int = 0
    d_min: int = 0
    canonical_id: str = ""
    canonical_hex: str = ""
    canonical_bitstring: str = ""
    window_avg_p_less: float = 0.0
    window_avg_dh: float = 0.0
    initial_rise_rate_avg: float = 0.0
    initial_rise_rate_max: float = 0.0
    quantum_time_sec: float = 0.0
    time_points: List[float] = field(default_factory=list)
    p_less_history: List[float] = field(default_factory=list)
    dh_history: List[float] = field(default_factory=list)
    p_blind: float = 0.0
    peak_p_less: float = 0.0
    peak_time: float = 0.0
    num_sampling_seeds: int = 1
    sample_seeds: List[int] = field(default_factory=list)
    sample_success_rates: List[float] = field(default_factory=list)
    sample_improved_shots: List[int] = field(default_factory=list)
    sample_total_shots: List[int] = field(default_factory=list)
    sample_best_energies: List[int] = field(default_factory=list)
    sample_mean_hamming_flips: List[float] = field(default_factory=list)
    best_d: int = 0
    best_d_rate: float = 0.0
    best_d_successes: int = 0
    best_d_trials: int = 0
    best_d_evals: int = 0
    rate_by_d: Dict[int, float] = field(default_factory=dict)
    trials_by_d: Dict[int, int] = field(default_factory=dict)
    evals_by_d: Dict[int, int] = field(default_factory=dict)
    kick_time_sec: float = 0.0
    restart_rate: float = 0.0
    restart_successes: int = 0
    restart_trials: int = 0
    restart_evals: int = 0
    restart_time_sec: float = 0.0
    tabu_direct_rate: float = 0.0
    tabu_direct_successes: int = 0
    tabu_direct_trials: int = 0
    tabu_direct_evals: int = 0
    tabu_direct_time_sec: float = 0.0
    tabu_kick_d: int = 0
    tabu_kick_rate: float = 0.0
    tabu_kick_successes: int = 0
    tabu_kick_trials: int = 0
    tabu_kick_evals: int = 0
    tabu_rate_by_d: Dict[int, float] = field(default_factory=dict)
    tabu_trials_by_d: Dict[int, int] = field(default_factory=dict)
    tabu_evals_by_d: Dict[int, int] = field(default_factory=dict)
    tabu_kick_time_sec: float = 0.0
    tabu_restart_rate: float = 0.0
    tabu_restart_successes: int = 0
    tabu_restart_trials: int = 0
    tabu_restart_evals: int = 0
    tabu_restart_time_sec: float = 0.0
    tabu_best_rate: float = 0.0
    tabu_best_method: str = ""
    sd_total_evaluations: int = 0
    tabu_total_evaluations: int = 0
    total_evaluations: int = 0


def window_average(time_points, p_less, t_start, avg_end):
    """Mean P_< over the points with t in [t_start, avg_end] (1e-9 slack), 0 if none
    (connector.cuh:817-829)."""
    s, c = 0.0, 0
    for t, p in zip(time_points, p_less):
        if t >= t_start - 1e-9 and t <= avg_end + 1e-9:
            s += p
            c += 1
    return s / c if c > 0 else 0.0


def window_end(t_start, k_sample_points, dt_sample, t_max):
    """avg_end of the window: the last sampling point when points are spaced by
    dt_sample, else t_max (connector.cuh:818-820)."""
    return t_start + (k_sample_points - 1) * dt_sample if (k_sample_points > 1 and dt_sample > 0.0) else t_max


def record_from_sampling(result, n, g, trap_rank, trap_bits, trap_energy, t_start=0.0, k_sample_points=20,
                         dt_sample=0.0, t_max=60.0, quantum_time_sec=0.0, d_min=0, **extra):
    """A TrapRecord from one `Engine.sampler_run` result, filled as the connector's
    run_quantum_simulation fills SingleTrapBenchmark (connector.cuh:647-678, 817-829).
    `extra` sets any other TrapRecord field (canonical ids, classical baselines)."""
    r = TrapRecord(n=n, g=float(g), trap_rank=int(trap_rank), trap_bits=int(trap_bits),
                   trap_energy=int(trap_energy), d_min=int(d_min))
    r.time_points = [float(x) for x in result["time_points"]]
    r.p_less_history = [float(x) for x in result["p_less_history"]]
    r.dh_history = [float(x) for x in result["dh_history"]]
    r.window_avg_dh = float(result["window_avg_dh"])
    r.initial_rise_rate_avg = float(result["initial_rise_rate_avg"])
    r.initial_rise_rate_max = float(result["initial_rise_rate_max"])
    if r.d_min == 0:
        r.d_min = int(result["d_min"])
    r.p_blind = float(result["p_blind"])
    r.peak_p_less = float(result["peak_p_less"])
    r.peak_time = float(result["peak_time"])
    stats = result.get("seed_stats", [])
    r.num_sampling_seeds = len(stats)
    r.sample_seeds = [int(s["seed"]) for s in stats]
    r.sample_success_rates = [float(s["success_rate"]) for s in stats]
    r.sample_improved_shots = [int(s["improved_shots"]) for s in stats]
    r.sample_total_shots = [int(s["total_shots_collected"]) for s in stats]
    r.sample_mean_hamming_flips = [float(s["mean_hamming_flips"]) for s in stats]
    r.sample_best_energies = [int(s["best_energy"]) for s in stats]
    r.window_avg_p_less = window_average(r.time_points, r.p_less_history, t_start,
                                         window_end(t_start, k_sample_points, dt_sample, t_max))
    r.quantum_time_sec = float(quantum_time_sec)
    for k, v in extra.items():
        if not hasattr(r, k):
            raise TypeError(f"unknown TrapRecord field {k}")
        setattr(r, k, v)
    return r


class _Stream:
    """The float-format state of a C++ ostream: floatfield (default, fixed,
    scientific), precision (6 at start) and the uppercase flag."""

    def __init__(self):
        self.parts = []
        self.mode = "default"
        self.prec = 6
        self.upper = False

    def fixed(self, p):
        self.mode, self.prec = "fixed", p
        return self

    def sci(self, p):
        self.mode, self.prec = "scientific", p
        return self

    def uppercase(self):
        self.upper = True
        return self

    def s(self, text):
        self.parts.append(text)
        return self

    def i(self, v):
        self.parts.append(str(int(v)))
        return self

    def hex(self, v):  # std::hex (and the uppercase flag) for one value, then std::dec
        t = format(int(v), "x")
        self.parts.append(t.upper() if self.upper else t)
        return self

    def f(self, v):
        v = float(v)
        if math.isnan(v):
            t = "-nan" if math.copysign(1.0, v) < 0 else "nan"
        elif math.isinf(v):
            t = "-inf" if v < 0 else "inf"
        elif self.mode == "fixed":
            t = "%.*f" % (self.prec, v)
        elif self.mode == "scientific":
            t = "%.*e" % (self.prec, v)
        else:
            t = "%.*g" % (self.prec if self.prec > 0 else 1, v)
        self.parts.append(t.upper() if self.upper else t)
        return self

    def text(self):
        return "".join(self.parts)


def time_series_csv(records):
    """The text of export_time_series_csv (connector.cuh:906-932)."""
    o = _Stream().s("N,g,trap_rank,trap_energy,time,p_less,dH,p_blind\n")
    for r in records:
        m = min(len(r.time_points), len(r.p_less_history))
        for i in range(m):
            dh = r.dh_history[i] if i < len(r.dh_history) else 0.0
            o.i(r.n).s(",").f(r.g).s(",").i(r.trap_rank).s(",").i(r.trap_energy).s(",")
            o.fixed(4).f(r.time_points[i]).s(",").sci(6).f(r.p_less_history[i]).s(",")
            o.fixed(4).f(dh).s(",").sci(6).f(r.p_blind).s("\n")
    return o.text()


RESULTS_HEADER = ("N,g,trap_rank,canonical_id,canonical_hex,trap_energy,d_min,window_avg_p_less,window_avg_dh,"
                  "initial_rise_rate_avg,initial_rise_rate_max,peak_p_less,peak_time,p_blind,"
                  "best_d,best_d_rate,best_d_successes,best_d_trials,best_d_evals,"
                  "restart_rate,restart_successes,restart_trials,restart_evals,"
                  "tabu_best_method,tabu_best_rate,tabu_direct_rate,tabu_kick_d,tabu_kick_rate,tabu_restart_rate,"
                  "sd_total_evaluations,tabu_total_evaluations,total_evaluations,"
                  "quantum_time_sec,kick_time_sec,restart_time_sec,tabu_kick_time_sec,"
                  "sample_seed1_rate,sample_seed2_rate,sample_seed3_rate,trap_bits\n")


def results_csv(records):
    """The text of export_results_csv (connector.cuh:839-904)."""
    o = _Stream().s(RESULTS_HEADER)
    for r in records:
        o.i(r.n).s(",").f(r.g).s(",").i(r.trap_rank).s(",").s(r.canonical_id).s(",").s(r.canonical_hex).s(",")
        o.i(r.trap_energy).s(",").i(r.d_min).s(",")
        o.sci(6).f(r.window_avg_p_less).s(",").fixed(4).f(r.window_avg_dh).s(",")
        o.sci(6).f(r.initial_rise_rate_avg).s(",").sci(6).f(r.initial_rise_rate_max).s(",")
        o.f(r.peak_p_less).s(",").fixed(4).f(r.peak_time).s(",").sci(6).f(r.p_blind).s(",")
        o.i(r.best_d).s(",").f(r.best_d_rate).s(",").i(r.best_d_successes).s(",").i(r.best_d_trials).s(",")
        o.i(r.best_d_evals).s(",").f(r.restart_rate).s(",").i(r.restart_successes).s(",")
        o.i(r.restart_trials).s(",").i(r.restart_evals).s(",")
        o.s('"').s(r.tabu_best_method).s('",').f(r.tabu_best_rate).s(",").f(r.tabu_direct_rate).s(",")
        o.i(r.tabu_kick_d).s(",").f(r.tabu_kick_rate).s(",").f(r.tabu_restart_rate).s(",")
        o.i(r.sd_total_evaluations).s(",").i(r.tabu_total_evaluations).s(",").i(r.total_evaluations).s(",")
        o.fixed(4).f(r.quantum_time_sec).s(",").f(r.kick_time_sec).s(",").f(r.restart_time_sec).s(",")
        o.f(r.tabu_kick_time_sec).s(",")
        for k in range(3):
            o.sci(6).f(r.sample_success_rates[k] if len(r.sample_success_rates) > k else 0.0).s(",")
        o.s("0x").uppercase().hex(r.trap_bits).s("\n")
    return o.text()


def _map_f(o, name, mp, indent):
    o.s(f'{indent}"{name}": {{')
    for di, k in enumerate(sorted(mp)):
        o.s(", " if di > 0 else "").s(f'"{int(k)}": ').sci(6).f(mp[k])
    o.s("},\n")


def _map_i(o, name, mp, indent):
    o.s(f'{indent}"{name}": {{')
    for di, k in enumerate(sorted(mp)):
        o.s(", " if di > 0 else "").s(f'"{int(k)}": ').i(mp[k])
    o.s("},\n")


def structured_json(records, n_override=0):
    """The text of export_structured_json (connector.cuh:934-1155): records grouped
    by (N, trap_rank) in ascending order, the first record of a group giving the
    trap and classical fields, every record of the group one g entry."""
    groups = {}
    for r in records:
        groups.setdefault((r.n, r.trap_rank), []).append(r)
    keys = sorted(groups)
    sys_n = n_override if n_override != 0 else (records[0].n if records else 0)
    o = _Stream()
    o.s("{\n").s('  "system": {\n').s('    "N": ').i(sys_n).s(",\n").s('    "num_seeds": ').i(len(keys)).s("\n")
    o.s("  },\n").s('  "seeds": [\n')
    for ti, key in enumerate(keys):
        lst = groups[key]
        a = lst[0]
        o.s("    {\n")
        o.s('      "N": ').i(a.n).s(",\n")
        o.s('      "trap_rank": ').i(a.trap_rank).s(",\n")
        o.s('      "canonical_id": "').s(a.canonical_id).s('",\n')
        o.s('      "canonical_hex": "').s(a.canonical_hex).s('",\n')
        o.s('      "canonical_bitstring": "').s(a.canonical_bitstring).s('",\n')
        o.s('      "trap_state_hex": "0x').uppercase().hex(a.trap_bits).s('",\n')
        o.s('      "trap_energy_E0": ').i(a.trap_energy).s(",\n")
        o.s('      "d_min": ').i(a.d_min).s(",\n")
        o.s('      "classical_baselines": {\n')
        c = "        "
        o.s(c + '"best_d": ').i(a.best_d).s(",\n")
        o.s(c + '"best_d_rate": ').sci(6).f(a.best_d_rate).s(",\n")
        o.s(c + '"best_d_successes": ').i(a.best_d_successes).s(",\n")
        o.s(c + '"best_d_trials": ').i(a.best_d_trials).s(",\n")
        o.s(c + '"best_d_evals": ').i(a.best_d_evals).s(",\n")
        _map_f(o, "rates_by_d", a.rate_by_d, c)
        _map_i(o, "trials_by_d", a.trials_by_d, c)
        _map_i(o, "evals_by_d", a.evals_by_d, c)
        o.s(c + '"restart_rate": ').sci(6).f(a.restart_rate).s(",\n")
        o.s(c + '"restart_successes": ').i(a.restart_successes).s(",\n")
        o.s(c + '"restart_trials": ').i(a.restart_trials).s(",\n")
        o.s(c + '"restart_evals": ').i(a.restart_evals).s(",\n")
        o.s(c + '"sd_total_evaluations": ').i(a.sd_total_evaluations).s(",\n")
        o.s(c + '"tabu_direct_rate": ').sci(6).f(a.tabu_direct_rate).s(",\n")
        o.s(c + '"tabu_direct_successes": ').i(a.tabu_direct_successes).s(",\n")
        o.s(c + '"tabu_direct_trials": ').i(a.tabu_direct_trials).s(",\n")
        o.s(c + '"tabu_direct_evals": ').i(a.tabu_direct_evals).s(",\n")
        o.s(c + '"tabu_kick_d": ').i(a.tabu_kick_d).s(",\n")
        o.s(c + '"tabu_kick_rate": ').sci(6).f(a.tabu_kick_rate).s(",\n")
        o.s(c + '"tabu_kick_successes": ').i(a.tabu_kick_successes).s(",\n")
        o.s(c + '"tabu_kick_trials": ').i(a.tabu_kick_trials).s(",\n")
        o.s(c + '"tabu_kick_evals": ').i(a.tabu_kick_evals).s(",\n")
        _map_f(o, "tabu_rates_by_d", a.tabu_rate_by_d, c)
        _map_i(o, "tabu_trials_by_d", a.tabu_trials_by_d, c)
        _map_i(o, "tabu_evals_by_d", a.tabu_evals_by_d, c)
        o.s(c + '"tabu_restart_rate": ').sci(6).f(a.tabu_restart_rate).s(",\n")
        o.s(c + '"tabu_restart_successes": ').i(a.tabu_restart_successes).s(",\n")
        o.s(c + '"tabu_restart_trials": ').i(a.tabu_restart_trials).s(",\n")
        o.s(c + '"tabu_restart_evals": ').i(a.tabu_restart_evals).s(",\n")
        o.s(c + '"tabu_best_rate": ').sci(6).f(a.tabu_best_rate).s(",\n")
        o.s(c + '"tabu_best_method": "').s(a.tabu_best_method).s('",\n')
        o.s(c + '"tabu_total_evaluations": ').i(a.tabu_total_evaluations).s(",\n")
        o.s(c + '"total_evaluations": ').i(a.total_evaluations).s(",\n")
        o.s(c + '"kick_time_sec": ').fixed(4).f(a.kick_time_sec).s(",\n")
        o.s(c + '"restart_time_sec": ').fixed(4).f(a.restart_time_sec).s(",\n")
        o.s(c + '"tabu_direct_time_sec": ').fixed(4).f(a.tabu_direct_time_sec).s(",\n")
        o.s(c + '"tabu_kick_time_sec": ').fixed(4).f(a.tabu_kick_time_sec).s(",\n")
        o.s(c + '"tabu_restart_time_sec": ').fixed(4).f(a.tabu_restart_time_sec).s("\n")
        o.s("      },\n")
        o.s('      "quantum_dynamics": {\n')
        q_ = "          "
        for gi, q in enumerate(lst):
            g_key = "%.2f" % q.g  # a fresh ostringstream: fixed, precision 2, no uppercase
            o.s(f'        "{g_key}": {{\n')
            o.s(q_ + '"g": ').fixed(2).f(q.g).s(",\n")
            o.s(q_ + '"window_avg_p_less": ').sci(6).f(q.window_avg_p_less).s(",\n")
            o.s(q_ + '"window_avg_dH": ').fixed(4).f(q.window_avg_dh).s(",\n")
            o.s(q_ + '"initial_rise_rate_avg": ').sci(6).f(q.initial_rise_rate_avg).s(",\n")
            o.s(q_ + '"initial_rise_rate_max": ').sci(6).f(q.initial_rise_rate_max).s(",\n")
            o.s(q_ + '"peak_p_less": ').sci(6).f(q.peak_p_less).s(",\n")
            o.s(q_ + '"peak_time": ').fixed(4).f(q.peak_time).s(",\n")
            o.s(q_ + '"p_blind": ').sci(6).f(q.p_blind).s(",\n")
            o.s(q_ + '"time_array": [')
            for ti2, t in enumerate(q.time_points):
                o.s(", " if ti2 > 0 else "").fixed(4).f(t)
            o.s("],\n").s(q_ + '"p_less_array": [')
            for ti2, p in enumerate(q.p_less_history):
                o.s(", " if ti2 > 0 else "").sci(6).f(p)
            o.s("],\n").s(q_ + '"dH_array": [')
            for ti2, d in enumerate(q.dh_history):
                o.s(", " if ti2 > 0 else "").fixed(4).f(d)
            o.s("],\n")
            o.s(q_ + '"quantum_time_sec": ').fixed(4).f(q.quantum_time_sec).s(",\n")
            o.s(q_ + '"sampling_validation": {\n')
            v = "            "
            o.s(v + '"num_sampling_seeds": ').i(q.num_sampling_seeds).s(",\n")
            o.s(v + '"seeds": [')
            for si, x in enumerate(q.sample_seeds):
                o.s(", " if si > 0 else "").i(x)
            o.s("],\n").s(v + '"sample_success_rates": [')
            for si, x in enumerate(q.sample_success_rates):
                o.s(", " if si > 0 else "").sci(6).f(x)
            o.s("],\n").s(v + '"sample_improved_shots": [')
            for si, x in enumerate(q.sample_improved_shots):
                o.s(", " if si > 0 else "").i(x)
            o.s("],\n").s(v + '"sample_total_shots": [')
            for si, x in enumerate(q.sample_total_shots):
                o.s(", " if si > 0 else "").i(x)
            o.s("],\n").s(v + '"sample_best_energies": [')
            for si, x in enumerate(q.sample_best_energies):
                o.s(", " if si > 0 else "").i(x)
            o.s("],\n").s(v + '"sample_mean_hamming_flips": [')
            for si, x in enumerate(q.sample_mean_hamming_flips):
                o.s(", " if si > 0 else "").fixed(4).f(x)
            o.s("]\n").s("          }\n")
            o.s("        }").s("," if gi + 1 < len(lst) else "").s("\n")
        o.s("      }\n")
        o.s("    }").s("," if ti + 1 < len(keys) else "").s("\n")
    o.s("  ]\n").s("}\n")
    return o.text()


def _write(path, text):
    d = os.path.dirname(path)
    if d:
        os.makedirs(d, exist_ok=True)
    with open(path, "w", newline="") as f:
        f.write(text)


def export_time_series_csv(path, records):
    _write(path, time_series_csv(records))


def export_results_csv(path, records):
    _write(path, results_csv(records))


def export_structured_json(path, records, n_override=0):
    _write(path, structured_json(records, n_override))
