"""ctypes bindings to the oracle libraries — TEST INFRASTRUCTURE ONLY.

``liboracle.so`` (trotter_oracle.cpp) is the complex128 CPU restatement of the
reference's sampler path; ``_ref/libbk_ref.so`` (ref_shim.cpp) is the reference's
own header-only energy / steepest-descent code, present only where the reference
tree was available at build time. Only tests/, __graft_entry__.smoke() and
bench.py's CPU legs may import this module.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None
_REF = None

u8p = ctypes.POINTER(ctypes.c_uint8)
u16p = ctypes.POINTER(ctypes.c_uint16)
u64p = ctypes.POINTER(ctypes.c_uint64)
i64p = ctypes.POINTER(ctypes.c_int64)
dp = ctypes.POINTER(ctypes.c_double)


def build():
    """Compile the oracle (and oracle/_ref when the reference tree is present)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        L.orc_labs_energy.restype = ctypes.c_int64
        L.orc_labs_energy.argtypes = [ctypes.c_int, ctypes.c_uint64]
        L.orc_labs_ck.argtypes = [ctypes.c_int, ctypes.c_uint64, i64p]
        L.orc_known_optimal_energy.restype = ctypes.c_int64
        L.orc_known_optimal_energy.argtypes = [ctypes.c_int]
        L.orc_canonical.restype = ctypes.c_uint64
        L.orc_canonical.argtypes = [ctypes.c_int, ctypes.c_uint64]
        L.orc_d_min.restype = ctypes.c_int
        L.orc_d_min.argtypes = [ctypes.c_int, ctypes.c_uint64, ctypes.c_int64, ctypes.c_int]
        L.orc_energy_table_u16.argtypes = [ctypes.c_int, u16p]
        L.orc_count_below.restype = ctypes.c_uint64
        L.orc_count_below.argtypes = [ctypes.c_int, ctypes.c_int64]
        L.orc_random_states.argtypes = [ctypes.c_int, ctypes.c_uint64, ctypes.c_int64, u64p]
        L.orc_steepest_descent.argtypes = [ctypes.c_int, ctypes.c_uint64, ctypes.c_uint64, u64p, i64p, u64p, i64p]
        L.orc_trotter_evolve.restype = ctypes.c_int
        L.orc_trotter_evolve.argtypes = [ctypes.c_int, ctypes.c_uint64, ctypes.c_int64, dp, ctypes.c_double,
                                         ctypes.c_double, ctypes.c_int, u8p, dp, dp, dp, ctypes.c_int, dp, dp]
        L.orc_trotter_adjoint.restype = ctypes.c_int
        L.orc_trotter_adjoint.argtypes = [ctypes.c_int, ctypes.c_uint64, ctypes.c_int64, dp, ctypes.c_double,
                                          ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int, dp, dp]
        L.orc_sample_indices.argtypes = [ctypes.c_int, dp, dp, ctypes.c_int64, u64p]
        L.orc_uniform_randoms.argtypes = [ctypes.c_uint64, ctypes.c_int64, dp]
        L.orc_sampler_run.restype = ctypes.c_int
        L.orc_sampler_run.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p]
        _LIB = L
    return _LIB


def ref_lib():
    """The reference's own compiled energy/descent code, or None when not built here."""
    global _REF
    if _REF is None:
        path = os.path.join(HERE, "_ref", "libbk_ref.so")
        if not os.path.exists(path):
            return None
        R = ctypes.CDLL(path)
        R.ref_calc_energy.restype = ctypes.c_int64
        R.ref_calc_energy.argtypes = [ctypes.c_int, ctypes.c_uint64]
        R.ref_calc_ck.argtypes = [ctypes.c_int, ctypes.c_uint64, i64p]
        R.ref_canonical.restype = ctypes.c_uint64
        R.ref_canonical.argtypes = [ctypes.c_int, ctypes.c_uint64]
        R.ref_d_min.restype = ctypes.c_int
        R.ref_d_min.argtypes = [ctypes.c_int, ctypes.c_uint64, ctypes.c_int64, ctypes.c_int]
        R.ref_known_optimal_energy.restype = ctypes.c_int64
        R.ref_known_optimal_energy.argtypes = [ctypes.c_int]
        R.ref_random_states.argtypes = [ctypes.c_int, ctypes.c_uint64, ctypes.c_int64, u64p]
        R.ref_steepest_descent.argtypes = [ctypes.c_int, ctypes.c_uint64, ctypes.c_uint64, u64p, i64p, u64p, i64p]
        _REF = R
    return _REF


def _ptr(a, t):
    return a.ctypes.data_as(t)


def labs_energy(n, bits):
    return int(lib().orc_labs_energy(n, bits))


def energy_table(n):
    out = np.empty(1 << n, dtype=np.uint16)
    lib().orc_energy_table_u16(n, _ptr(out, u16p))
    return out


def count_below(n, e0):
    return int(lib().orc_count_below(n, e0))


def d_min(n, bits, target=-1, max_d=-1):
    return int(lib().orc_d_min(n, bits, target, max_d))


def canonical(n, bits):
    return int(lib().orc_canonical(n, bits))


def random_states(n, seed, count):
    out = np.empty(count, dtype=np.uint64)
    lib().orc_random_states(n, seed, count, _ptr(out, u64p))
    return out


def steepest_descent(n, start, max_evals=0, use_ref=False):
    L = ref_lib() if use_ref else lib()
    fn = L.ref_steepest_descent if use_ref else L.orc_steepest_descent
    fs, fe, ev, st = ctypes.c_uint64(), ctypes.c_int64(), ctypes.c_uint64(), ctypes.c_int64()
    fn(n, start, max_evals, ctypes.byref(fs), ctypes.byref(fe), ctypes.byref(ev), ctypes.byref(st))
    return int(fs.value), int(fe.value), int(ev.value), int(st.value)


def known_optimal_energy(n):
    return int(lib().orc_known_optimal_energy(n))


def select_trap(n, seed, n_descents, quantile, use_ref=None):
    """Trap policy of the benchmark configurations (the lowest `quantile` of
    `n_descents` seeded descents, global optima excluded, first minimum in
    generation order at or below the threshold energy), restated on the
    reference's descent: starts mt19937_64(seed) & mask
    (classical.cuh:557-604), single-flip steepest descent (:625-712).
    use_ref=None takes the reference's own compiled code when oracle/_ref was
    built, else the oracle's restatement of it; both are bit-exact."""
    if use_ref is None:
        use_ref = ref_lib() is not None
    if use_ref:
        R = ref_lib()
        starts = np.empty(n_descents, dtype=np.uint64)
        R.ref_random_states(n, seed, n_descents, _ptr(starts, u64p))
    else:
        starts = random_states(n, seed, n_descents)
    finals = [steepest_descent(n, int(x), 0, use_ref=use_ref)[:2] for x in starts]
    opt = known_optimal_energy(n)
    kept = sorted(e for _, e in finals if opt < 0 or e > opt)
    if not kept:
        raise ValueError(f"every descent at n = {n} reached a global optimum")
    thr = kept[int(np.floor(quantile * (len(kept) - 1)))]
    for bits, e in finals:
        if (opt < 0 or e > opt) and e <= thr:
            return bits, e
    raise ValueError("no trap at or below the threshold")


def uniform_randoms(seed, count):
    out = np.empty(count, dtype=np.float64)
    lib().orc_uniform_randoms(seed, count, _ptr(out, dp))
    return out


def trotter_evolve(n, s0, e0, g, dt, n_steps, measure=None, diag_scale=0.0, threads=0, want_state=False,
                   step_seconds=None):
    """Complex128 restatement of the reference step loop; returns (p_less, d_h, norm[, state]).

    ``step_seconds`` (optional float64 array of n_steps) receives the wall time of each step."""
    g_arr = np.ascontiguousarray(np.broadcast_to(np.asarray(g, dtype=np.float64), (max(n_steps, 1),)))
    if measure is None:
        flags = np.ones(n_steps + 1, dtype=np.uint8)
    else:
        flags = np.zeros(n_steps + 1, dtype=np.uint8)
        flags[np.asarray(measure, dtype=np.int64)] = 1
    m = int(flags.sum())
    p = np.zeros(m)
    d = np.zeros(m)
    nn = np.zeros(m)
    st = np.zeros(2 << n) if want_state else None
    rc = lib().orc_trotter_evolve(n, s0, e0, _ptr(g_arr, dp), dt, diag_scale, n_steps, _ptr(flags, u8p),
                                  _ptr(p, dp), _ptr(d, dp), _ptr(nn, dp), threads,
                                  _ptr(st, dp) if want_state else None,
                                  _ptr(step_seconds, dp) if step_seconds is not None else None)
    if rc != 0:
        raise ValueError(f"orc_trotter_evolve rejected n={n}, n_steps={n_steps}")
    if want_state:
        return p, d, nn, st[0::2] + 1j * st[1::2]
    return p, d, nn


def segment_steps(n_steps, n_segments):
    """Step -> segment map of a piecewise-constant schedule with equal segments."""
    if n_segments <= 0 or n_steps % n_segments:
        raise ValueError("n_steps must be a multiple of n_segments")
    return np.repeat(np.arange(n_segments), n_steps // n_segments)


def trotter_adjoint(n, s0, e0, g, dt, n_steps, objective=0, diag_scale=0.0, threads=0):
    """Adjoint gradient of O(T) (0: P_<, 1: <d_H>) w.r.t. the per-step field g_k.

    Returns (O, dO/dg_k for k < n_steps); complex128, exact gates."""
    g_arr = np.ascontiguousarray(np.broadcast_to(np.asarray(g, dtype=np.float64), (max(n_steps, 1),)))
    grad = np.zeros(max(n_steps, 1))
    val = np.zeros(1)
    rc = lib().orc_trotter_adjoint(n, s0, e0, _ptr(g_arr, dp), dt, diag_scale, n_steps, objective, threads,
                                   _ptr(val, dp), _ptr(grad, dp))
    if rc != 0:
        raise ValueError(f"orc_trotter_adjoint rejected n={n}, n_steps={n_steps}, objective={objective}")
    return float(val[0]), grad[:n_steps]


def sample_indices(n, state, randnums):
    st = np.empty(2 << n)
    st[0::2] = state.real
    st[1::2] = state.imag
    r = np.ascontiguousarray(randnums, dtype=np.float64)
    out = np.empty(len(r), dtype=np.uint64)
    lib().orc_sample_indices(n, _ptr(st, dp), _ptr(r, dp), len(r), _ptr(out, u64p))
    return out


class SamplerConfig(ctypes.Structure):
    """Mirror of orc_sampler_config (reference SamplerConfig, src/sampling/sampler.cuh:235-260)."""
    _fields_ = [("n", ctypes.c_int32), ("num_sample_points", ctypes.c_int32),
                ("shots_per_point", ctypes.c_int32), ("num_sampling_seeds", ctypes.c_int32),
                ("track_p_less", ctypes.c_int32), ("record_trajectory", ctypes.c_int32),
                ("seed", ctypes.c_uint64), ("seed_stride", ctypes.c_uint64),
                ("g", ctypes.c_double), ("dt", ctypes.c_double), ("t_max", ctypes.c_double),
                ("t_start", ctypes.c_double), ("dt_sample", ctypes.c_double), ("dt_trajectory", ctypes.c_double)]


class _Result(ctypes.Structure):
    _fields_ = [("n_points", ctypes.c_int64), ("time_points", dp), ("p_less_history", dp), ("dh_history", dp),
                ("start_energy", ctypes.c_int64), ("d_min", ctypes.c_int32),
                ("p_blind", ctypes.c_double), ("peak_p_less", ctypes.c_double), ("peak_time", ctypes.c_double),
                ("window_avg_dh", ctypes.c_double), ("initial_rise_rate_avg", ctypes.c_double),
                ("initial_rise_rate_max", ctypes.c_double),
                ("total_shots_collected", ctypes.c_uint64), ("improved_shots", ctypes.c_uint64),
                ("total_evals", ctypes.c_uint64), ("unique_basis_size", ctypes.c_uint64),
                ("success_rate", ctypes.c_double), ("per_eval_rate", ctypes.c_double),
                ("mean_hamming_flips", ctypes.c_double), ("n_seeds", ctypes.c_int32),
                ("seed_values", u64p), ("seed_total_shots", u64p), ("seed_improved_shots", u64p),
                ("seed_success_rate", dp), ("seed_mean_hamming", dp), ("seed_best_energy", i64p)]


def sampler_run(cfg: dict, start_bits: int) -> dict:
    """Reference ISampler::sample() semantics on the complex128 restatement (small n only)."""
    c = SamplerConfig(**cfg)
    T = int(round(c.t_max / c.dt))
    ns = max(1, c.num_sampling_seeds)
    bufs = {k: np.zeros(T + 1) for k in ("time_points", "p_less_history", "dh_history")}
    sb = {k: np.zeros(ns, dtype=np.uint64) for k in ("seed_values", "seed_total_shots", "seed_improved_shots")}
    sd = {k: np.zeros(ns) for k in ("seed_success_rate", "seed_mean_hamming")}
    sbe = np.zeros(ns, dtype=np.int64)
    r = _Result()
    for k, v in bufs.items():
        setattr(r, k, _ptr(v, dp))
    for k, v in sb.items():
        setattr(r, k, _ptr(v, u64p))
    for k, v in sd.items():
        setattr(r, k, _ptr(v, dp))
    r.seed_best_energy = _ptr(sbe, i64p)
    rc = lib().orc_sampler_run(ctypes.byref(c), start_bits, ctypes.byref(r))
    if rc != 0:
        raise ValueError("orc_sampler_run rejected the configuration")
    npt = r.n_points
    out = {k: getattr(r, k) for k, _ in _Result._fields_ if not k.startswith("seed_") and k not in bufs}
    for k, v in bufs.items():
        out[k] = v[:npt].copy()
    out["seed_stats"] = [dict(seed=int(sb["seed_values"][i]), total_shots_collected=int(sb["seed_total_shots"][i]),
                              improved_shots=int(sb["seed_improved_shots"][i]),
                              success_rate=float(sd["seed_success_rate"][i]),
                              mean_hamming_flips=float(sd["seed_mean_hamming"][i]),
                              best_energy=int(sbe[i])) for i in range(ns)]
    return out


def fullspace_matvec(n, g, x, scale=None, threads=0):
    """y = (scale E - g sum_j X_j) x, the reference's per-state order (diagonalizer.cuh:60-77)."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.empty_like(x)
    dp = ctypes.POINTER(ctypes.c_double)
    L = lib()
    L.orc_fullspace_matvec.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, dp, dp, ctypes.c_int]
    if L.orc_fullspace_matvec(n, g, (1.0 / n) if scale is None else scale, _ptr(x, dp), _ptr(y, dp), threads):
        raise ValueError("orc_fullspace_matvec rejected its arguments")
    return y


def fullspace_lanczos(n, g, max_krylov_dim=100, tolerance=1e-12, normalize_by_n=True, threads=0):
    """The reference's plain Lanczos (diagonalizer.cuh:418-482) on the CPU: (alphas, betas)."""
    dp = ctypes.POINTER(ctypes.c_double)
    L = lib()
    L.orc_fullspace_lanczos.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                        ctypes.c_double, dp, dp, ctypes.POINTER(ctypes.c_int), ctypes.c_int]
    a = np.zeros(max(max_krylov_dim, 1))
    b = np.zeros(max(max_krylov_dim, 1))
    m = ctypes.c_int(0)
    if L.orc_fullspace_lanczos(n, g, (1.0 / n) if normalize_by_n else 1.0, max_krylov_dim, tolerance, _ptr(a, dp),
                               _ptr(b, dp), ctypes.byref(m), threads):
        raise ValueError("orc_fullspace_lanczos rejected its arguments")
    return a[:m.value].copy(), b[:max(m.value - 1, 0)].copy()
