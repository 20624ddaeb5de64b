#!/usr/bin/env python3
"""Benchmark: Trotter amplitude-steps per second of the transverse-field LABS
evolution at N = 28 on B200 (complex64 fused engine), the reference sampler's
headline configuration ("Large N": one deep trap from the lowest 1% of 4000
seeded steepest descents, g = 0.35, dt = 0.02, P_< and <d_H> every 20 steps).

One bench step = `--trotter` Trotter steps (default 100, i.e. 5 measurement
intervals) run through bk_evolve from the trap state; K steps cover 2000
Trotter steps at the defaults, the configuration's full run.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Multi-GPU (launched by torchrun, one rank per GPU): independent replicas, each
rank evolves its own trap (seed 42 + rank); no collective on the data path
(weak scaling). `value` = all ranks' amp-steps / the slowest rank's device time.

`--impl reference` times the reference's own algorithm (phase kernel, then one
2x2 Rx per qubit, complex128) as restated on the host CPU in oracle/ (the
reference's cuStateVec code cannot be built here), all host threads, one
Trotter step per bench step. Under torchrun only rank 0 runs it.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG_ROOT = os.path.join(ROOT, "bernasconi-krylov_b200")
for _p in (ROOT, PKG_ROOT):
    if _p not in sys.path:
        sys.path.insert(0, _p)

METRIC = "Trotter amp-steps/s at N={n}"
UNIT = "amp-steps/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--n", type=int, default=28)
    ap.add_argument("--precision", choices=["c64", "c128"], default="c64")
    ap.add_argument("--trotter", type=int, default=100, help="Trotter steps per bench step")
    ap.add_argument("--measure-every", type=int, default=20)
    ap.add_argument("--g", type=float, default=0.35)
    ap.add_argument("--dt", type=float, default=0.02)
    ap.add_argument("--cpu-baseline-steps", type=int, default=2)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-compare", action="store_true")
    ap.add_argument("--engine-mode", type=int, default=None,
                    help="0 persistent, 1 one launch per pass, 2 A1 launch + fused strided launch, "
                         "3 the same with the fused strided pass in two self-served groups")
    ap.add_argument("--workload", choices=["large", "batched", "adjoint", "matvec"], default="large",
                    help="large: the N=28 headline; batched: 512 instances (64 traps x 8 g), N in {16,18,20,22}")
    ap.add_argument("--slab-lag", type=int, default=None)
    ap.add_argument("--split-w2", type=int, default=None, help="qubits of the S2 pass (0 = default split)")
    ap.add_argument("--a1-kernel", type=int, default=None, choices=[0, 1, 2, 3],
                    help="per-pass A1 kernel: 0 = 256x16, 1 = 512x8, 2 = warp-local (element bits 0-8), "
                         "3 = warp-local over 32 KB half tiles")
    ap.add_argument("--phase-table", type=int, default=None, choices=[0, 1],
                    help="complex64 A1 kernels 1-3: 1 = the full per-energy phase table")
    ap.add_argument("--no-tune", action="store_true", help="engine defaults instead of the autotuner's choice")
    ap.add_argument("--adjoint-config", choices=["standard", "large"], default="standard",
                    help="adjoint workload: standard = N=22, 1280 steps; large = N=28, 2000 steps")
    ap.add_argument("--kernel-table-steps", type=int, default=3,
                    help="bench steps of the separate per-kernel timing pass (roofline)")
    return ap.parse_args()


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    except Exception:
        return 6650.0, "fallback (6650 GB/s copy bandwidth; MEASURED_PEAKS.json absent)"


def committed_traffic():
    """DRAM bytes per launch of the dominant kernel from the committed ncu summary, if any."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            return json.load(f)
    except Exception:
        return {}


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms during the timed region."""

    def __init__(self, index):
        self.index = index
        self.samples = []
        self.proc = None

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            # nvidia-smi's start-up can hold the driver for seconds; let it settle
            # before the timed region so it cannot stall a timed launch
            t0 = time.time()
            while not self.samples and time.time() - t0 < 15:
                time.sleep(0.05)
            self.samples.clear()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) == 7:
                self.samples.append(parts)

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if s[3 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def large_config(a, n, bits, e0, seed, world=1):
    """The workload of the N = 28 headline line, shared by both arms so the
    driver compares like with like."""
    S = 8 if a.precision == "c64" else 16
    return {"workload": f"N={n} single trap (lowest 1% of 4000 descents, seed {seed}), g={a.g}, dt={a.dt}, "
                        f"{a.trotter} Trotter steps per bench step, P_< and <d_H> every {a.measure_every} steps",
            "n": n, "trap_bits": hex(bits), "trap_energy": int(e0), "trotter_steps_per_step": a.trotter,
            "l2": f"state {((1 << n) * S) / 2**30:.1f} GiB > 126 MB L2, no flush needed",
            "parallelism": f"replicas x{world}"}


def oracle_trap(n, seed=42):
    """The benchmark trap selected by the oracle (the reference's compiled descent
    when oracle/_ref was built): the CPU legs never load the product library."""
    from oracle import oracle as O
    return O.select_trap(n, seed, 4000 if n >= 28 else 1000, 0.01 if n >= 28 else 0.05)


def cpu_baseline(n, steps, g, dt):
    """The oracle's complex128 per-qubit restatement of the reference step, all host threads."""
    from oracle import oracle as O
    bits, e0 = oracle_trap(n)
    secs = np.zeros(steps)
    threads = os.cpu_count() or 1
    O.trotter_evolve(n, bits, e0, g, dt, steps, measure=[0], threads=threads, step_seconds=secs)
    return {"value": (1 << n) / float(np.mean(secs)), "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{steps} Trotter steps of the N={n} trap in complex128 on the host "
                      f"(oracle/trotter_oracle.cpp: phase + {n} per-qubit Rx passes per step, OpenMP), "
                      f"mean step time {np.mean(secs):.3f} s"}


def ed_baseline(sizes=(8, 10, 12), g=0.35, points=41, dt=0.5):
    """The reference's CPU fallback for small N (dense exact diagonalisation,
    connector.cuh:683-805 on Eigen, absent here) restated with numpy/LAPACK
    (oracle/ed_oracle.py): eigh of the 2^N x 2^N Hamiltonian and `points`
    propagated time points, timed on the host's cores."""
    from oracle import oracle as O
    from oracle import ed_oracle
    out = {}
    for n in sizes:
        bits = int(O.steepest_descent(n, 12345 % (1 << n))[0])
        e0 = O.labs_energy(n, bits)
        t0 = time.perf_counter()
        ed_oracle.propagate(n, g, bits, e0, np.arange(points) * dt, O.energy_table(n))
        out[str(n)] = {"seconds": time.perf_counter() - t0, "time_points": points}
    return {"kind": "numpy/LAPACK restatement (Eigen absent)", "cores": os.cpu_count(), "sizes": out}


def run_reference(a):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import oracle as O
    n = a.n
    bits, e0 = oracle_trap(n)
    total = a.warmup + a.steps
    secs = np.zeros(total)
    threads = os.cpu_count() or 1
    meas = [k for k in range(0, total + 1) if k % a.measure_every == 0]
    O.trotter_evolve(n, bits, e0, a.g, a.dt, total, measure=meas, threads=threads, step_seconds=secs)
    timed = secs[a.warmup:]
    v = (1 << n) * len(timed) / float(timed.sum())
    line = {"metric": METRIC.format(n=n), "value": v, "unit": UNIT, "impl": "reference", "n_gpus": a.gpus,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": 1e3 * float(timed.mean()),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c128",
            "data": "synthetic (seeded trap from 4000 steepest descents, no dataset)",
            "config": large_config(a, n, bits, e0, 42, a.gpus),
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": f"a bounded sample of the workload: {total} Trotter steps of the same N={n} "
                                       f"trap ({a.warmup} untimed), one per bench step, P_< and <d_H> every "
                                       f"{a.measure_every} steps, by the oracle's complex128 restatement of the "
                                       f"reference's phase + per-qubit Rx loop on all host threads"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "custatevec": custatevec_probe()}
    print(json.dumps(line))


def custatevec_probe():
    """Whether the reference's own GPU path (cuStateVec, sampler.cuh:412-707) could
    run on this machine: the cuquantum Python package or a libcustatevec the
    loader can find. The reference sampler also needs custatevec.h to build."""
    import ctypes.util
    found = []
    try:
        import cuquantum  # noqa: F401
        found.append("python package cuquantum")
    except Exception:
        pass
    lib = ctypes.util.find_library("custatevec")
    if lib:
        found.append(lib)
    hdr = [d for d in ("/usr/include", "/usr/local/include", "/usr/local/cuda/include")
           if os.path.exists(os.path.join(d, "custatevec.h"))]
    if found and hdr:
        return {"available": True, "found": found + hdr}
    return {"available": False,
            "detail": "unavailable on this box: " + ("; ".join(found) if found else "no cuquantum package, no "
                      "libcustatevec") + ("" if hdr else ", no custatevec.h")}


def replica_trap(n, rank, n_descents=4000, quantile=0.01):
    """Trap of one replica: the lowest `quantile` of `n_descents` seeded descents, seed 42 + rank."""
    import bk_b200 as bk
    return bk.select_trap(n, 42 + rank, n_descents, quantile)


def max_over_ranks(x, world, device):
    """Largest value over all ranks (the job's time is its slowest rank's)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_value(units_per_rank, world, seconds_max):
    """Weak scaling: every rank processes units_per_rank; the job ends with its slowest rank."""
    return units_per_rank * world / seconds_max


def tuned_knobs(eng, a, n, prec, trap):
    """Engine knobs for this run: explicit flags, else the autotuner's cached choice
    for this device and size, else a tuning sweep now (not timed, not cached)."""
    from bk_b200 import tune
    explicit = {k: v for k, v in (("engine_mode", a.engine_mode), ("slab_lag", a.slab_lag),
                                  ("split_w2", a.split_w2), ("a1_wide", a.a1_kernel),
                                  ("phase_table", a.phase_table)) if v is not None}
    if explicit or a.no_tune:
        for k, v in explicit.items():
            eng.set_option(k, v)
        return dict(source="flags" if explicit else "engine defaults", **explicit)
    best = tune.apply(eng, n, prec)
    if best is not None:
        return dict(source="autotuner cache (bk_b200/tuning/b200.json)", **best)
    entry = tune.tune(eng, n, prec, steps=10, warmup=2, trap=trap, write=False)
    return dict(source="autotuner sweep at start-up (untimed)", **entry["best"])


def batched_instances(seed=2024):
    """64 traps (seeded descents, lowest 5% of 1000) with N drawn from {16,18,20,22}, x 8 g in [0.2, 0.5]."""
    import bk_b200 as bk
    rng = np.random.default_rng(seed)
    traps = []
    for j in range(64):
        n = int(rng.choice([16, 18, 20, 22]))
        bits, e0 = bk.select_trap(n, 42 + j, 1000, 0.05)
        traps.append((n, bits, e0))
    return [dict(n=n, s0=bits, e0=e0, g=float(g)) for (n, bits, e0) in traps for g in np.linspace(0.2, 0.5, 8)]


def run_batched(a):
    import torch
    import bk_b200 as bk
    steps_t = 500
    dev = torch.device("cuda", 0)
    eng = bk.Engine(0)
    inst = batched_instances()
    amp_steps = float(sum(1 << d["n"] for d in inst)) * steps_t
    stream = torch.cuda.ExternalStream(eng.stream_handle(), device=dev)
    meas = range(0, steps_t + 1)
    from bk_b200 import tune
    lag = tune.batch_lag(eng, inst)
    lag_src = "autotuner cache (bk_b200/tuning/b200.json)"
    if lag is None:
        lag = tune.tune_batch(eng, inst, a.dt, steps_t, measure=meas, write=False)["best"]["lag"]
        lag_src = "autotuner sweep at start-up (untimed)"
    for _ in range(max(a.warmup, 1)):
        eng.evolve_batch(inst, a.dt, steps_t, measure=meas, precision=bk.BK_C64, use_graph=True, lag=lag)
    torch.cuda.synchronize(dev)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(0) as clocks:
        t0 = time.perf_counter()
        ev0.record(stream)
        for _ in range(a.steps):
            p, d, nn = eng.evolve_batch(inst, a.dt, steps_t, measure=meas, precision=bk.BK_C64, use_graph=True,
                                        lag=lag)
        ev1.record(stream)
        torch.cuda.synchronize(dev)
        wall = time.perf_counter() - t0
    dev_s = ev0.elapsed_time(ev1) / 1e3
    value = amp_steps * a.steps / dev_s
    # the same 512 instances one after another, each through its own launches
    seq = {}
    for mode in (1, 0):
        eng.set_option("engine_mode", mode)
        eng.evolve(inst[0]["n"], inst[0]["s0"], inst[0]["g"], a.dt, 4, measure=[0], e0=inst[0]["e0"])
        torch.cuda.synchronize(dev)
        e0_, e1_ = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0_.record(stream)
        for d in inst:
            eng.evolve(d["n"], d["s0"], d["g"], a.dt, steps_t, measure=meas, e0=d["e0"], precision=bk.BK_C64)
        e1_.record(stream)
        torch.cuda.synchronize(dev)
        seq["sequential_" + ("one_launch_per_pass" if mode == 1 else "persistent_per_instance")] = \
            amp_steps / (e0_.elapsed_time(e1_) / 1e3)
    best_seq = max(seq.values())
    # roofline: one persistent launch per bench step runs all 500 steps of all
    # 512 instances; algorithmic bytes 32 per amplitude-step (two complex64
    # read + write passes), timed by the CUDA events bracketing the launches
    peak, peak_kind = measured_peaks()
    launch_s = dev_s / a.steps
    alg = 32.0 * amp_steps
    roof = {"bound": "hbm", "kernel": "persist_kernel (batched, one graph launch per bench step)",
            "achieved": alg / launch_s / 1e9, "peak": peak, "unit": "GB/s", "frac": alg / launch_s / 1e9 / peak,
            "peak_source": peak_kind, "algorithmic_bytes_per_launch": alg, "avg_launch_ms": 1e3 * launch_s,
            "traffic": None,
            "l2": "each statevector is 0.5-32 MiB (N = 16-22, complex64); the tasks of a few statevectors in flight "
                  "fit the 126 MB L2, so part of the traffic is served from L2 and the HBM fraction is nominal"}
    line = {"metric": "Batched Trotter amp-steps/s (512 instances, N in {16,18,20,22}, complex64)", "value": value,
            "unit": UNIT, "n_gpus": 1, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": 1e3 * dev_s / a.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "c64",
            "data": "synthetic (64 seeded traps x 8 g, no dataset)",
            "config": {"workload": "512 instances = 64 traps (lowest 5% of 1000 descents, N uniform in "
                                   "{16,18,20,22}, seed 2024) x 8 g in linspace(0.2, 0.5, 8); dt=0.02, 500 Trotter "
                                   "steps, P_< and <d_H> every step; one persistent launch through a captured "
                                   "CUDA graph per bench step",
                       "instances": len(inst), "trotter_steps_per_step": steps_t,
                       "tuning": {"lag": lag, "source": lag_src},
                       "amp_steps_per_step": amp_steps},
            "compare": dict(seq, batched_over_best_sequential=value / best_seq),
            "e2e": {"value": amp_steps * a.steps / wall, "unit": UNIT, "h2d_bytes_per_step": 24 * len(inst) + 501,
                    "d2h_bytes_per_step": 3 * 8 * len(inst) * 501},
            "clocks": clocks.summary(), "roofline": roof, "gpu_launches": a.steps,
            "check": {"p_less_mean_last": float(np.mean(p[:, -1])), "norm_max_dev": float(np.max(np.abs(nn - 1)))}}
    eng.close()
    if not a.no_cpu_baseline:
        line["cpu_baseline"] = batched_cpu_baseline(inst, a.dt)
    print(json.dumps(line))


def batched_cpu_baseline(inst, dt, per_n=2, steps=10):
    """The oracle's complex128 restatement on the same instance mix, sampled:
    `per_n` instances of each N in the batch, `steps` Trotter steps each, all host threads."""
    from oracle import oracle as O
    threads = os.cpu_count() or 1
    picked, seen = [], {}
    for d in inst:
        if seen.get(d["n"], 0) < per_n:
            seen[d["n"]] = seen.get(d["n"], 0) + 1
            picked.append(d)
    amp, t0 = 0.0, time.perf_counter()
    for d in picked:
        O.trotter_evolve(d["n"], d["s0"], d["e0"], d["g"], dt, steps, measure=[0], threads=threads)
        amp += float(1 << d["n"]) * steps
    secs = time.perf_counter() - t0
    return {"value": amp / secs, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{len(picked)} instances of the batch ({per_n} per N in {sorted(seen)}), {steps} Trotter steps "
                      f"each, oracle complex128 restatement (phase + per-qubit Rx), {secs:.1f} s"}


def run_adjoint(a):
    """Adjoint gradient. standard: N=22 trap (lowest 5% of 1000 descents), 64 segments g_j ~ U[0.25, 0.45],
    dt=0.02, 1280 steps, checkpoints every 128. large: N=28 trap (lowest 1% of 4000 descents), 40 segments of
    50 steps (2000 steps), checkpoint interval from bk_adjoint's free-memory rule. One bench step = one
    bk_adjoint call (value and all segment gradients)."""
    import torch
    import bk_b200 as bk
    large = a.adjoint_config == "large"
    n, nseg, T, K = (28, 40, 2000, 0) if large else (22, 64, 1280, 128)
    prec = bk.BK_C64 if a.precision == "c64" else bk.BK_C128
    dev = torch.device("cuda", 0)
    eng = bk.Engine(0)
    bits, e0 = bk.select_trap(n, 42, 4000, 0.01) if large else bk.select_trap(n, 42, 1000, 0.05)
    gs = np.random.default_rng(2028 if large else 42).uniform(0.25, 0.45, nseg)
    g_steps = np.repeat(gs, T // nseg)
    stream = torch.cuda.ExternalStream(eng.stream_handle(), device=dev)
    # complex64: the reverse A1 pass takes the diagonal phase from the full per-energy table (measured faster)
    eng.set_option("phase_table", 1 if a.phase_table is None else a.phase_table)
    for _ in range(max(a.warmup, 1)):
        eng.adjoint(n, bits, gs, a.dt, T, e0=e0, precision=prec, checkpoint_every=K)
    torch.cuda.synchronize(dev)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    fw, rv = [], []
    with ClockSampler(0) as clocks:
        t0 = time.perf_counter()
        ev0.record(stream)
        for _ in range(a.steps):
            val, grad, st = eng.adjoint(n, bits, gs, a.dt, T, e0=e0, precision=prec, checkpoint_every=K)
            fw.append(st["forward_ms"])
            rv.append(st["reverse_ms"])
        ev1.record(stream)
        torch.cuda.synchronize(dev)
        wall = time.perf_counter() - t0
    dev_s = ev0.elapsed_time(ev1) / 1e3
    # one plain forward run of the same schedule (measurement at T only)
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    for _ in range(a.steps):
        eng.evolve(n, bits, g_steps, a.dt, T, measure=[T], e0=e0, precision=prec)
    f1.record(stream)
    torch.cuda.synchronize(dev)
    fwd_s = f0.elapsed_time(f1) / 1e3 / a.steps
    amp_steps = float(1 << n) * T
    # roofline of the reverse sweep (the dominant part): per amplitude-step it
    # reads and writes psi and lambda in two passes, 8 S bytes (S = 8 complex64, 16 complex128)
    S = 8 if prec == bk.BK_C64 else 16
    peak, peak_kind = measured_peaks()
    rev_s = float(np.mean(rv)) / 1e3
    alg = 8.0 * S * amp_steps
    roof = {"bound": "hbm", "kernel": "adjoint reverse sweep (dual-state tile passes)",
            "achieved": alg / rev_s / 1e9, "peak": peak, "unit": "GB/s", "frac": alg / rev_s / 1e9 / peak,
            "peak_source": peak_kind, "algorithmic_bytes_per_launch": alg, "avg_launch_ms": 1e3 * rev_s,
            "traffic": None,
            "l2": ("psi and lambda are 2 GiB each at N = 28 complex64, far above L2" if large else
                   "psi and lambda are 32 MiB each at N = 22 complex64: both fit the 126 MB L2, so the HBM "
                   "fraction is nominal")}
    cpu = None
    if not a.no_cpu_baseline:
        from oracle import oracle as O
        threads = os.cpu_count() or 1
        Tc = 2 if large else 20
        # the oracle's adjoint takes n <= 26: the large configuration is sampled at N = 26 (its own trap)
        nc = min(n, 26)
        bc, ec = (bits, e0) if nc == n else O.select_trap(nc, 42, 200, 0.01)
        t0c = time.perf_counter()
        O.trotter_adjoint(nc, bc, ec, g_steps[:Tc], a.dt, Tc, threads=threads)
        secs = time.perf_counter() - t0c
        what = f"the same N={n} trap and schedule" if nc == n else f"an N={nc} trap with the same schedule"
        cpu = {"value": float(1 << nc) * Tc / secs, "unit": UNIT, "cores": threads, "kind": "port",
               "sample": f"forward + adjoint gradient of {Tc} steps of {what} by the oracle (complex128, exact "
                         f"gates, sqrt(T) checkpoints), {secs:.1f} s"}
    cfg_name = (f"N={n}, {nseg} segments, {T} steps" + (", checkpoints sized to free HBM" if large else ""))
    line = {"metric": f"Adjoint gradient amp-steps/s ({cfg_name}; forward + reverse sweep)",
            "value": amp_steps * a.steps / dev_s, "unit": UNIT, "n_gpus": 1, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": 1e3 * dev_s / a.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": a.precision, "data": "synthetic (seeded trap and field schedule, no dataset)",
            "config": {"workload": (f"N={n} trap (lowest 1% of 4000 descents, seed 42), {nseg} segments g_j ~ "
                                    "U[0.25, 0.45] (seed 2028), dt=0.02, 2000 steps, checkpoint interval from the "
                                    "free-memory rule, objective P_<(T)") if large else
                                   ("N=22 trap (lowest 5% of 1000 descents, seed 42), 64 segments g_j ~ U[0.25, 0.45] "
                                    "(seed 42), dt=0.02, 1280 steps, checkpoints every 128, objective P_<(T)"),
                       "n": n, "segments": nseg, "trotter_steps": T, "checkpoint_every": st["checkpoint_every"],
                       "n_checkpoints": st["n_checkpoints"],
                       "l2": ("statevectors of 2 GiB (complex64) each, far above the 126 MB L2" if large else
                              "two 32 MiB statevectors (complex64) fit the 126 MB L2")},
            "compare": {"forward_ms": 1e3 * fwd_s, "gradient_ms": 1e3 * dev_s / a.steps,
                        "gradient_cost_in_forwards": dev_s / a.steps / fwd_s,
                        "reverse_over_forward": float(np.mean(rv)) / float(np.mean(fw)),
                        "max_checkpoint_drift": st["max_drift"]},
            "e2e": {"value": amp_steps * a.steps / wall, "unit": UNIT, "h2d_bytes_per_step": 8 * nseg + 96,
                    "d2h_bytes_per_step": 8 * (nseg + 1 + T)},
            "clocks": clocks.summary(), "roofline": roof, "cpu_baseline": cpu,
            "check": {"p_less_T": val, "grad_max_abs": float(np.max(np.abs(grad)))}}
    eng.close()
    print(json.dumps(line))


def run_matvec(a):
    """Full-space Hamiltonian matvec (the Lanczos hot loop): y = (E/N - g sum_j X_j) x over all 2^N states in
    FP64 at N = 28 (vectors 2 GiB each, > L2); one bench step = 10 products."""
    import torch
    import bk_b200 as bk
    from oracle import oracle as O
    n = a.n if a.n else 28
    reps = 10
    dev = torch.device("cuda", 0)
    eng = bk.Engine(0)
    x = torch.from_numpy(np.random.default_rng(42).standard_normal(1 << n)).to(dev)
    y = torch.empty_like(x)
    stream = torch.cuda.ExternalStream(eng.stream_handle(), device=dev)
    for _ in range(max(a.warmup, 3)):
        eng.fullspace_matvec(n, 0.35, x, y)
    torch.cuda.synchronize(dev)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(0) as clocks:
        ev0.record(stream)
        for _ in range(a.steps * reps):
            eng.fullspace_matvec(n, 0.35, x, y)
        ev1.record(stream)
        torch.cuda.synchronize(dev)
    dev_s = ev0.elapsed_time(ev1) / 1e3
    # per-pass times from a separate pass with CUDA events around every launch
    eng.set_kernel_timing(True)
    for _ in range(reps):
        eng.fullspace_matvec(n, 0.35, x, y)
    torch.cuda.synchronize(dev)
    kt = eng.kernel_timing()
    eng.set_kernel_timing(False)
    # the reference's one-thread-per-state form on the same vectors
    for _ in range(2):
        eng.fullspace_matvec(n, 0.35, x, y, method=bk.BK_PLAIN)
    p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    p0.record(stream)
    for _ in range(reps):
        eng.fullspace_matvec(n, 0.35, x, y, method=bk.BK_PLAIN)
    p1.record(stream)
    torch.cuda.synchronize(dev)
    plain_per = p0.elapsed_time(p1) / 1e3 / reps
    # end to end through the public call with host buffers: pinned x in, y out, per product
    hx = x.cpu().pin_memory()
    hy = torch.empty_like(hx).pin_memory()
    t0 = time.perf_counter()
    for _ in range(a.steps):
        xd = hx.to(dev, non_blocking=True)
        eng.fullspace_matvec(n, 0.35, xd, y)
        hy.copy_(y, non_blocking=True)
        torch.cuda.synchronize(dev)
    e2e_s = (time.perf_counter() - t0) / a.steps
    states = float(1 << n)
    per = dev_s / (a.steps * reps)
    peak, peak_kind = measured_peaks()
    alg = 18.0 * states  # x and y once (8 B each) and E once (2 B) per product
    fb_, ft_ = kt.get("fs_block", (0, 0.0)), kt.get("fs_tile", (0, 0.0))
    fs = (fb_[0] + ft_[0], fb_[1] + ft_[1])
    # CPU baseline: the oracle's per-state restatement (OpenMP, all host cores) at N = 24
    nc, xc = 24, np.random.default_rng(1).standard_normal(1 << 24)
    O.fullspace_matvec(nc, 0.35, xc)
    c0 = time.perf_counter()
    for _ in range(3):
        O.fullspace_matvec(nc, 0.35, xc)
    cpu_rate = 3 * float(1 << nc) / (time.perf_counter() - c0)
    line = {"metric": f"Full-space H matvec states/s (N={n}, FP64, Lanczos hot loop)",
            "value": states / per, "unit": "states/s", "n_gpus": 1, "steps": a.steps, "warmup": max(a.warmup, 3),
            "ms_per_step": 1e3 * dev_s / a.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic (seeded Gaussian vector, no dataset)",
            "config": {"workload": f"y = (E/N) x - 0.35 sum_j x[i ^ 2^j] over 2^{n} states, FP64, 10 products per "
                                   "bench step", "n": n, "products_per_step": reps,
                       "l2": f"x and y {8 * states / 2**30:.1f} GiB each > 126 MB L2, no flush needed",
                       "passes": "block pass over 8192-state blocks (index bits 0-12 in shared memory, bits 13-22 "
                                 "as L2 sweeps of partner blocks), then for n > 23 one strided tile pass over "
                                 "bits [23, n) (each tile one tensor-map box)",
                       "design_dram_bytes_per_state": 42},
            "roofline": {"bound": "hbm", "kernel": "fs_block + fs_tile (all passes of one product)",
                         "achieved": alg / per / 1e9,
                         "peak": peak, "unit": "GB/s", "frac": alg / per / 1e9 / peak, "peak_source": peak_kind,
                         "algorithmic_bytes_per_launch": alg, "avg_launch_ms": 1e3 * per, "traffic": None,
                         "block_pass_avg_ms": fb_[1] / max(fb_[0], 1), "strided_pass_avg_ms": ft_[1] / max(ft_[0], 1)},
            "cpu_baseline": {"value": cpu_rate, "unit": "states/s", "cores": os.cpu_count(), "kind": "port",
                             "sample": "3 products at N = 24 by the oracle's per-state restatement "
                                       "(oracle/trotter_oracle.cpp orc_fullspace_matvec, OpenMP)"},
            "e2e": {"value": states / e2e_s, "unit": "states/s", "h2d_bytes_per_step": int(8 * states),
                    "d2h_bytes_per_step": int(8 * states)},
            "compare": {"plain_states_per_s": states / plain_per, "plain_ms": 1e3 * plain_per,
                        "tiled_over_plain": plain_per / per},
            "gpu_launches": int(fs[0]), "clocks": clocks.summary()}
    eng.close()
    print(json.dumps(line))


def main():
    a = parse()
    if a.impl == "reference":
        run_reference(a)
        return
    if a.workload == "batched":
        run_batched(a)
        return
    if a.workload == "adjoint":
        run_adjoint(a)
        return
    if a.workload == "matvec":
        run_matvec(a)
        return
    import torch
    import torch.distributed as dist
    import bk_b200 as bk

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=torch.device("cuda", local))

    def barrier():
        if world > 1:
            dist.barrier()


    n, T = a.n, a.trotter
    prec = bk.BK_C64 if a.precision == "c64" else bk.BK_C128
    eng = bk.Engine(local)
    bits, e0 = replica_trap(n, rank)
    tuning = tuned_knobs(eng, a, n, prec, (bits, e0))
    meas = list(range(0, T + 1, a.measure_every))
    dev = torch.device("cuda", local)
    stream = torch.cuda.ExternalStream(eng.stream_handle(), device=dev)

    def bench_step():
        return eng.evolve(n, bits, a.g, a.dt, T, measure=meas, e0=e0, precision=prec)

    for _ in range(max(a.warmup, 0)):
        bench_step()

    # ---- device-timed region (value): the production path, no per-launch events ----
    barrier()
    torch.cuda.synchronize(dev)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clocks:
        ev0.record(stream)
        for _ in range(a.steps):
            p_last, d_last, n_last = bench_step()
        ev1.record(stream)
        torch.cuda.synchronize(dev)
    barrier()
    dev_s = ev0.elapsed_time(ev1) / 1e3
    dev_s_max = max_over_ranks(dev_s, world, f"cuda:{local}")

    # ---- per-kernel table for the roofline: a separate pass with CUDA events
    # around every launch (outside the timed region above) ----
    barrier()
    eng.set_kernel_timing(True)
    for _ in range(min(a.steps, a.kernel_table_steps)):
        bench_step()
    torch.cuda.synchronize(dev)
    timing = eng.kernel_timing()
    eng.set_kernel_timing(False)
    barrier()

    # ---- end-to-end region: the C-ABI call with host buffers, wall clock ----
    barrier()
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    for _ in range(a.steps):
        bench_step()
    torch.cuda.synchronize(dev)
    barrier()
    e2e_s = max_over_ranks(time.perf_counter() - t0, world, f"cuda:{local}")

    amp_steps = float(1 << n) * T * a.steps * world
    value = whole_job_value(float(1 << n) * T * a.steps, world, dev_s_max)
    e2e = whole_job_value(float(1 << n) * T * a.steps, world, e2e_s)

    # ---- roofline of the dominant kernel ----
    S = 8 if prec == bk.BK_C64 else 16
    # algorithmic bytes per launch: a pass reads and writes the state once (2 S per
    # amplitude); one persistent launch runs all T Trotter steps of a call (4 S per
    # amplitude-step: two such passes per step)
    per_launch_bytes = {"measure": S, "plain_phase": 2 * S, "plain_rx": 2 * S, "persist": 4 * S * T,
                        "tile_a1": 2 * S, "tile_s2": 2 * S, "tile_s3": 2 * S, "tile_m": S}
    dom = max(timing.items(), key=lambda kv: kv[1][1])
    dname, (dl, dms) = dom
    abytes = per_launch_bytes.get(dname, 2 * S) * float(1 << n)
    achieved = abytes / (dms / dl / 1e3) / 1e9
    peak, peak_kind = measured_peaks()
    traffic = committed_traffic().get(f"{dname}/n{n}/{a.precision}")
    # launches per bench step from the timing pass, scaled to the timed steps
    # (+ one basis-state init per call)
    table_steps = max(1, min(a.steps, a.kernel_table_steps))
    launches = int(round(sum(v[0] for v in timing.values()) * a.steps / table_steps)) + a.steps

    line = {"metric": METRIC.format(n=n), "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": 1e3 * dev_s_max / a.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "c64" if prec == bk.BK_C64 else "c128",
            "data": "synthetic (seeded trap from 4000 steepest descents, no dataset)",
            "config": large_config(a, n, bits, e0, 42 + rank, world), "tuning": tuning,
            "roofline": {"bound": "hbm", "kernel": dname, "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_source": peak_kind,
                         "algorithmic_bytes_per_launch": abytes, "avg_launch_ms": dms / dl,
                         "traffic": traffic,
                         # the whole Trotter step against the two-round-trip model (4 S bytes per amplitude-step)
                         "step": {"algorithmic_bytes": 4.0 * S * float(1 << n),
                                  "ms": 1e3 * dev_s_max / (a.steps * T),
                                  "achieved": 4.0 * S * float(1 << n) / (dev_s_max / (a.steps * T)) / 1e9,
                                  "frac": 4.0 * S * float(1 << n) / (dev_s_max / (a.steps * T)) / 1e9 / peak}},
            "kernels": {k: {"launches": v[0], "total_ms": round(v[1], 3)} for k, v in timing.items()},
            "kernel_table": f"{table_steps} bench steps with CUDA events around every launch, after the timed "
                            "region (the timed region runs without them)",
            "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": 8 * 8 + (T + 1),
                    "d2h_bytes_per_step": 8 * 3 * len(meas) + 8 * 4 * len(meas)},
            "gpu_launches": launches, "clocks": clocks.summary(),
            "check": {"p_less_last": float(p_last[-1]), "d_h_last": float(d_last[-1]),
                      "norm_last": float(n_last[-1])}}

    if rank == 0 and world == 1 and not a.no_compare:
        from bk_b200 import tune
        cmp = {}
        # the complex128 runs use complex128's own tuned knobs (else the engine defaults)
        if tune.apply(eng, n, bk.BK_C128) is None:
            tune.apply_config(eng, tune.DEFAULTS)
        c128_series = None
        for name, pr, meth, steps in (("c128_fused", bk.BK_C128, bk.BK_FUSED, T),
                                      ("c128_plain", bk.BK_C128, bk.BK_PLAIN, 20)):
            eng.evolve(n, bits, a.g, a.dt, 2, measure=[0], e0=e0, precision=pr, method=meth)
            torch.cuda.synchronize(dev)
            e0_ = torch.cuda.Event(enable_timing=True)
            e1_ = torch.cuda.Event(enable_timing=True)
            e0_.record(stream)
            out = eng.evolve(n, bits, a.g, a.dt, steps, measure=list(range(0, steps + 1, a.measure_every)), e0=e0,
                             precision=pr, method=meth)
            e1_.record(stream)
            torch.cuda.synchronize(dev)
            cmp[name] = float(1 << n) * steps / (e0_.elapsed_time(e1_) / 1e3)
            if name == "c128_fused":
                c128_series = out
        cmp["c64_fused"] = value
        cmp["c64_fused_over_c128_plain"] = value / cmp["c128_plain"]
        cmp["c64_fused_over_c128_fused"] = value / cmp["c128_fused"]
        cmp["custatevec"] = custatevec_probe()
        line["compare"] = cmp
        if prec == bk.BK_C64 and c128_series is not None:
            # the bench step's own series (c64, tuned knobs) against complex128 on the same trap and schedule
            p128, d128, _ = c128_series
            line["check"]["c64_vs_c128"] = {
                "trotter_steps": T, "points": len(meas),
                "max_abs_dP_less": float(np.max(np.abs(p_last - p128))),
                "max_abs_d_dH": float(np.max(np.abs(d_last - d128))),
                "bar_dP_less": 1e-6}
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        try:
            line["cpu_baseline"] = cpu_baseline(n, a.cpu_baseline_steps, a.g, a.dt)
            line["cpu_baseline"]["ed_dense"] = ed_baseline()
        except Exception as exc:  # report, do not hide
            line["cpu_baseline"] = {"value": None, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
                                    "sample": f"failed: {exc}"}
    eng.close()
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
