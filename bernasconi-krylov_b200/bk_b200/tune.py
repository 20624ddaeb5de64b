"""Autotuner of the tile engine's schedule (the reference has no tuner: its
mixer is N cuStateVec calls per step, sampler.cuh:611-617).

Knobs (engine options, include/bk_engine.h):
  engine_mode  0 = persistent dataflow kernel (every step in one launch, A1 tiles
               handed to S2 through L2), 1 = one grid launch per pass, 2 = the
               A1 pass as a grid launch and both strided passes in one
               persistent launch (S3 re-reads S2's slabs from L2), 3 = mode 2
               with the fused launch served by two self-loading groups;
  slab_lag     persistent engines: slabs between a slab's A1 and S2 tasks (mode
               0), or between a slab's S2 and S3 tasks (mode 2);
  split_w2     qubits of the S2 pass (the rest go to S3), 0 = engine default;
  e_source     E(s) for the diagonal phase: 0 = uint16 table, 1 = recomputed
               from popcounts in the pass (no E traffic, more arithmetic);
  a1_wide      per-pass schedule, the A1 kernel: 0 = 256 threads x 16 elements
               (element bits 0-11), 1 = 512 x 8, 2 = warp-local (element bits
               0-8 inside each warp, no CTA barrier; the strided passes take
               bits 9 and up; up to 27 element bits), 3 = warp-local with
               4-warp CTAs over 32 KB half tiles (four CTAs per SM);
  phase_table  complex64 per-pass A1 kernels: 1 = the diagonal phase of
               each energy level from a full table (E = floor(n/2) mod 4 for
               every LABS energy) as two half-angle shear rotations, 0 = level
               table and residual polynomials.
For the batched engine the knob is the task-block lag between a statevector
slab's A1 and S2 tasks.

Each candidate is timed with CUDA events on the engine's stream over `steps`
Trotter steps after `warmup` (the state of a large N is far larger than L2, so
no flush is needed); the fastest is kept. Results are cached as JSON per device
(name and SM count) and per (precision, N) — or batch signature — together
with every measurement, so the choice can be audited. The committed cache
``tuning/b200.json`` holds the results of ``python -m bk_b200.tune`` on a B200.
"""
import argparse
import json
import os


from ._lib import BK_C64, BK_C128

DEFAULT_CACHE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tuning", "b200.json")
KNOBS = ("engine_mode", "slab_lag", "split_w2", "e_source", "a1_wide", "phase_table")
DEFAULTS = {"engine_mode": 0, "slab_lag": 3, "split_w2": 0, "e_source": 0, "a1_wide": 0, "phase_table": 0}
ELEM_BITS = 12  # element bits of one 64 KB tile


def device_key(device=0):
    import torch
    p = torch.cuda.get_device_properties(device)
    return f"{p.name}/{p.multi_processor_count}sm"


def entry_key(n, precision):
    return f"{'c64' if precision == BK_C64 else 'c128'}/n{n}"


def default_w2(rest):
    return rest if rest <= 9 else (rest + 1) // 2


def candidates(n, precision):
    """Engine mode x slab lag x S2 width (the default split and its neighbours)."""
    np_ = n - 1 if precision == BK_C64 else n
    rest = np_ - ELEM_BITS
    if rest < 1:
        return [dict(DEFAULTS)]
    d = default_w2(rest)
    widths = [0] + [w for w in (d - 1, d + 1) if 1 <= w <= 9 and w <= rest and rest - w <= 9]
    out = []
    for w in widths:
        for wide in (0, 1):
            out.append(dict(engine_mode=1, slab_lag=3, split_w2=w, e_source=0, a1_wide=wide))
        for lag in (1, 2, 3, 4, 6):
            out.append(dict(engine_mode=0, slab_lag=lag, split_w2=w, e_source=0, a1_wide=0))
    # warp-local A1 (per-pass): np - 9 strided bits, the default split and its neighbours
    rest9 = np_ - 9
    if 1 <= rest9 <= 18:
        d9 = default_w2(rest9)
        for w in [0] + [w for w in (d9 - 1, d9 + 1) if 3 <= w <= 9 and w <= rest9 and rest9 - w <= 9]:
            for wide in (2, 3):
                out.append(dict(engine_mode=1, slab_lag=3, split_w2=w, e_source=0, a1_wide=wide))
    # fused strided pass (mode 2: S2 and S3 in one launch, S3 reading S2's slabs
    # from L2), for each A1 kernel and split that leaves a third pass to fuse
    def fused(rest_bits, ws, wides):
        for w in ws:
            w2 = w if w else default_w2(rest_bits)
            if rest_bits - w2 < 1:
                continue
            for wide in wides:
                for lag in (1, 2, 3):
                    out.append(dict(engine_mode=2, slab_lag=lag, split_w2=w, e_source=0, a1_wide=wide))
                out.append(dict(engine_mode=3, slab_lag=2, split_w2=w, e_source=0, a1_wide=wide))
    fused(rest, widths, (0, 1))
    if 1 <= rest9 <= 18:
        fused(rest9, [0] + [w for w in (d9 - 1, d9 + 1) if 3 <= w <= 9 and w <= rest9 and rest9 - w <= 9], (2, 3))
    # complex64: the full phase table with every per-pass candidate whose A1 kernel takes it (1-3)
    if precision == BK_C64:
        out += [dict(c, phase_table=1) for c in list(out) if c["engine_mode"] in (1, 2, 3)]
    # E recomputed in the pass, on the default split of both schedules
    out.append(dict(engine_mode=1, slab_lag=3, split_w2=0, e_source=1, a1_wide=0))
    out.append(dict(engine_mode=0, slab_lag=3, split_w2=0, e_source=1, a1_wide=0))
    return out


def _timer(eng):
    import torch
    stream = torch.cuda.ExternalStream(eng.stream_handle())

    def run(fn):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        fn()
        b.record(stream)
        b.synchronize()
        return a.elapsed_time(b) / 1e3
    return run


def apply_config(eng, cfg):
    for k in KNOBS:
        eng.set_option(k, int(cfg.get(k, DEFAULTS[k])))


def measure(eng, n, precision, cfg, bits, e0, steps=20, warmup=4, g=0.35, dt=0.02):
    """amp-steps/s of one configuration."""
    apply_config(eng, cfg)
    meas = list(range(0, steps + 1, 20))
    eng.evolve(n, bits, g, dt, warmup, measure=[0], e0=e0, precision=precision)
    sec = _timer(eng)(lambda: eng.evolve(n, bits, g, dt, steps, measure=meas, e0=e0, precision=precision))
    return float(1 << n) * steps / sec


def load_cache(path=None):
    path = path or DEFAULT_CACHE
    if os.path.exists(path):
        with open(path) as f:
            return json.load(f)
    return {}


def save_cache(cache, path=None):
    path = path or DEFAULT_CACHE
    os.makedirs(os.path.dirname(path), exist_ok=True)
    with open(path, "w") as f:
        json.dump(cache, f, indent=1, sort_keys=True)
        f.write("\n")


def tune(eng, n, precision=BK_C64, steps=20, warmup=4, cache_path=None, trap=None, write=True):
    """Times every candidate for (n, precision); returns the best entry and caches it."""
    from ._lib import select_trap
    bits, e0 = trap if trap is not None else select_trap(n, 42, 200, 0.01)
    results = []
    for cfg in candidates(n, precision):
        results.append(dict(cfg, amp_steps_per_s=measure(eng, n, precision, cfg, bits, e0, steps, warmup)))
    best = max(results, key=lambda r: r["amp_steps_per_s"])
    entry = {"best": {k: best[k] for k in KNOBS}, "amp_steps_per_s": best["amp_steps_per_s"],
             "steps": steps, "candidates": results}
    if write:
        cache = load_cache(cache_path)
        cache.setdefault(device_key(eng.device), {})[entry_key(n, precision)] = entry
        save_cache(cache, cache_path)
    apply_config(eng, entry["best"])
    return entry


def apply(eng, n, precision=BK_C64, cache_path=None):
    """Sets the cached best knobs for (device, n, precision); returns them or None."""
    cache = load_cache(cache_path)
    entry = cache.get(device_key(eng.device), {}).get(entry_key(n, precision))
    if entry is None:
        return None
    apply_config(eng, entry["best"])
    return entry["best"]


def batch_key(instances, precision):
    ns = sorted(d["n"] for d in instances)
    return f"batch/{'c64' if precision == BK_C64 else 'c128'}/{len(ns)}x{'-'.join(map(str, sorted(set(ns))))}"


def tune_batch(eng, instances, dt, n_steps, measure=None, precision=BK_C64, lags=(1, 2, 3, 4, 6, 8), cache_path=None,
               write=True):
    """Times the batched engine for each task-block lag; returns and caches the best."""
    results = []
    t = _timer(eng)
    for lag in lags:
        eng.evolve_batch(instances, dt, n_steps, measure=measure, precision=precision, use_graph=True, lag=lag)
        sec = t(lambda: eng.evolve_batch(instances, dt, n_steps, measure=measure, precision=precision,
                                         use_graph=True, lag=lag))
        results.append(dict(lag=lag, amp_steps_per_s=float(sum(1 << d["n"] for d in instances)) * n_steps / sec))
    best = max(results, key=lambda r: r["amp_steps_per_s"])
    entry = {"best": {"lag": best["lag"]}, "amp_steps_per_s": best["amp_steps_per_s"], "candidates": results}
    if write:
        cache = load_cache(cache_path)
        cache.setdefault(device_key(eng.device), {})[batch_key(instances, precision)] = entry
        save_cache(cache, cache_path)
    return entry


def batch_lag(eng, instances, precision=BK_C64, cache_path=None):
    entry = load_cache(cache_path).get(device_key(eng.device), {}).get(batch_key(instances, precision))
    return None if entry is None else entry["best"]["lag"]


def main(argv=None):
    from ._lib import Engine
    ap = argparse.ArgumentParser(description="tune the tile engine's schedule and cache the result")
    ap.add_argument("--n", type=int, nargs="+", default=[24, 26, 28, 30])
    ap.add_argument("--precision", nargs="+", choices=["c64", "c128"], default=["c64", "c128"])
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--cache", default=None)
    args = ap.parse_args(argv)
    eng = Engine(0)
    for pr in args.precision:
        prec = BK_C64 if pr == "c64" else BK_C128
        for n in args.n:
            if prec == BK_C128 and n > 30:
                continue
            e = tune(eng, n, prec, steps=args.steps, cache_path=args.cache)
            print(json.dumps({"precision": pr, "n": n, "best": e["best"], "amp_steps_per_s": e["amp_steps_per_s"]}),
                  flush=True)
    eng.close()


if __name__ == "__main__":
    main()
