"""ctypes marshalling for include/bk_engine.h."""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)

BK_OK, BK_ERR_INVALID, BK_ERR_CUDA, BK_ERR_OOM, BK_ERR_TIMEOUT, BK_ERR_NORM, BK_ERR_UNSUPPORTED, \
    BK_ERR_NO_DEVICE = range(8)
BK_C64, BK_C128 = 0, 1
BK_FUSED, BK_PLAIN = 0, 1
BK_ORDER_REFERENCE, BK_ORDER_STRANG = 0, 1
BK_OBJ_P_LESS, BK_OBJ_D_H = 0, 1

_u8p = ctypes.POINTER(ctypes.c_uint8)
_u16p = ctypes.POINTER(ctypes.c_uint16)
_u64p = ctypes.POINTER(ctypes.c_uint64)
_i64p = ctypes.POINTER(ctypes.c_int64)
_dp = ctypes.POINTER(ctypes.c_double)
_LIB = None


class BkError(RuntimeError):
    def __init__(self, status, msg=""):
        self.status = status
        super().__init__(f"bk status {status}: {msg}")


class EvolveParams(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int32), ("precision", ctypes.c_int32), ("method", ctypes.c_int32),
                ("ordering", ctypes.c_int32), ("s0", ctypes.c_uint64), ("e0", ctypes.c_int64),
                ("dt", ctypes.c_double), ("diag_scale", ctypes.c_double), ("n_steps", ctypes.c_int32),
                ("reserved0", ctypes.c_int32), ("g", _dp), ("g_const", ctypes.c_double),
                ("measure", _u8p), ("norm_tol", ctypes.c_double), ("sample", _u8p), ("shots", ctypes.c_int32),
                ("reserved1", ctypes.c_int32), ("randnums", _dp), ("samples_out", _u64p)]


class BatchInstanceC(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int32), ("reserved", ctypes.c_int32), ("s0", ctypes.c_uint64), ("e0", ctypes.c_int64),
                ("g_const", ctypes.c_double), ("g", _dp)]


class BatchParamsC(ctypes.Structure):
    _fields_ = [("precision", ctypes.c_int32), ("n_steps", ctypes.c_int32), ("dt", ctypes.c_double),
                ("diag_scale", ctypes.c_double), ("measure", _u8p), ("use_graph", ctypes.c_int32),
                ("lag", ctypes.c_int32)]


class AdjointParamsC(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int32), ("precision", ctypes.c_int32), ("s0", ctypes.c_uint64), ("e0", ctypes.c_int64),
                ("dt", ctypes.c_double), ("diag_scale", ctypes.c_double), ("n_steps", ctypes.c_int32),
                ("n_segments", ctypes.c_int32), ("g", _dp), ("segment_of_step", ctypes.POINTER(ctypes.c_int32)),
                ("checkpoint_every", ctypes.c_int32), ("objective", ctypes.c_int32)]


class AdjointStatsC(ctypes.Structure):
    _fields_ = [("value", ctypes.c_double), ("norm", ctypes.c_double), ("checkpoint_every", ctypes.c_int32),
                ("n_checkpoints", ctypes.c_int32), ("max_drift", ctypes.c_double), ("forward_ms", ctypes.c_double),
                ("reverse_ms", ctypes.c_double)]


class LanczosParamsC(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int32), ("g", ctypes.c_double), ("num_eigenpairs", ctypes.c_int32),
                ("max_krylov_dim", ctypes.c_int32), ("tolerance", ctypes.c_double), ("normalize_by_n", ctypes.c_int32),
                ("alphas", ctypes.POINTER(ctypes.c_double)), ("betas", ctypes.POINTER(ctypes.c_double))]


class LanczosStatsC(ctypes.Structure):
    _fields_ = [("krylov_dim", ctypes.c_int32), ("matvecs", ctypes.c_int32), ("seconds", ctypes.c_double)]


class MinimumFamilyC(ctypes.Structure):
    _fields_ = [("id", ctypes.c_uint64), ("canonical_state", ctypes.c_uint64), ("sample_state", ctypes.c_uint64),
                ("energy", ctypes.c_int64), ("times_visited", ctypes.c_uint64),
                ("evals_to_first_find", ctypes.c_uint64)]


class CollectStatsC(ctypes.Structure):
    _fields_ = [("total_starts", ctypes.c_uint64), ("total_evals", ctypes.c_uint64), ("batches", ctypes.c_uint64),
                ("saturated", ctypes.c_int32), ("reserved", ctypes.c_int32)]


class SamplerConfigC(ctypes.Structure):
    """bk_sampler_config — the reference's SamplerConfig (sampler.cuh:235-260) plus precision/method."""
    _fields_ = [("n", ctypes.c_int32), ("num_sample_points", ctypes.c_int32), ("shots_per_point", ctypes.c_int32),
                ("num_sampling_seeds", ctypes.c_int32), ("track_p_less", ctypes.c_int32),
                ("record_trajectory", ctypes.c_int32), ("verbose", ctypes.c_int32), ("precision", ctypes.c_int32),
                ("method", ctypes.c_int32), ("reserved", ctypes.c_int32), ("seed", ctypes.c_uint64),
                ("seed_stride", ctypes.c_uint64), ("g", ctypes.c_double), ("dt", ctypes.c_double),
                ("t_max", ctypes.c_double), ("t_start", ctypes.c_double), ("dt_sample", ctypes.c_double),
                ("dt_trajectory", ctypes.c_double)]


class SeedStatsC(ctypes.Structure):
    _fields_ = [("seed", ctypes.c_uint64), ("total_shots_collected", ctypes.c_uint64),
                ("improved_shots", ctypes.c_uint64), ("success_rate", ctypes.c_double),
                ("per_eval_rate", ctypes.c_double), ("mean_hamming_flips", ctypes.c_double),
                ("best_energy", ctypes.c_int64)]


class SamplingResultC(ctypes.Structure):
    _fields_ = [("unique_basis", _u64p), ("unique_basis_size", ctypes.c_int64),
                ("total_shots_collected", ctypes.c_uint64), ("improved_shots", ctypes.c_uint64),
                ("success_rate", ctypes.c_double), ("per_eval_rate", ctypes.c_double),
                ("total_evals", ctypes.c_uint64), ("mean_hamming_flips", ctypes.c_double),
                ("seed_stats", ctypes.POINTER(SeedStatsC)), ("n_seed_stats", ctypes.c_int32),
                ("d_min", ctypes.c_int32), ("time_points", _dp), ("p_less_history", _dp), ("dh_history", _dp),
                ("n_points", ctypes.c_int64), ("window_avg_dh", ctypes.c_double),
                ("initial_rise_rate_avg", ctypes.c_double), ("initial_rise_rate_max", ctypes.c_double),
                ("start_energy", ctypes.c_int64), ("p_blind", ctypes.c_double), ("peak_p_less", ctypes.c_double),
                ("peak_time", ctypes.c_double)]


def library_path():
    return os.path.join(PKG, "lib", "libbk_b200.so")


def load_library(build_if_missing=True):
    """Load the engine library (building it in-tree with nvcc if it is missing)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    path = library_path()
    if not os.path.exists(path) and build_if_missing:
        import importlib.util
        spec = importlib.util.spec_from_file_location("bk_build", os.path.join(PKG, "build.py"))
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        mod.build()
    L = ctypes.CDLL(path)
    c_ctx = ctypes.c_void_p
    L.bk_abi_version.restype = ctypes.c_int
    L.bk_status_string.restype = ctypes.c_char_p
    L.bk_status_string.argtypes = [ctypes.c_int]
    L.bk_last_error.restype = ctypes.c_char_p
    L.bk_last_error.argtypes = [c_ctx]
    L.bk_create.argtypes = [ctypes.c_int, ctypes.POINTER(c_ctx)]
    L.bk_destroy.argtypes = [c_ctx]
    L.bk_labs_energy.argtypes = [ctypes.c_int, _u64p, ctypes.c_int64, _i64p]
    L.bk_energy_table.argtypes = [c_ctx, ctypes.c_int, _u16p]
    L.bk_p_blind.argtypes = [c_ctx, ctypes.c_int, ctypes.c_int64, _u64p, _dp]
    L.bk_evolve.argtypes = [c_ctx, ctypes.POINTER(EvolveParams), _dp, _dp, _dp]
    L.bk_export_state.argtypes = [c_ctx, _dp]
    L.bk_set_kernel_timing.argtypes = [c_ctx, ctypes.c_int]
    L.bk_kernel_timing.argtypes = [c_ctx, ctypes.c_int, ctypes.POINTER(ctypes.c_char_p), _i64p, _dp]
    L.bk_sample.argtypes = [c_ctx, _dp, ctypes.c_int64, _u64p]
    L.bk_stream.argtypes = [c_ctx, ctypes.POINTER(ctypes.c_void_p)]
    L.bk_set_option.argtypes = [c_ctx, ctypes.c_int, ctypes.c_int64]
    L.bk_evolve_batch.argtypes = [c_ctx, ctypes.POINTER(BatchParamsC), ctypes.POINTER(BatchInstanceC), ctypes.c_int32,
                                  _dp, _dp, _dp]
    L.bk_get_option.argtypes = [c_ctx, ctypes.c_int, _i64p]
    L.bk_steepest_descent_gpu.argtypes = [c_ctx, ctypes.c_int, _u64p, ctypes.c_int64, ctypes.c_uint64, _u64p, _i64p,
                                          _u64p]
    L.bk_collect_minima.argtypes = [c_ctx, ctypes.c_int, ctypes.c_uint64, ctypes.c_int64, ctypes.c_int64,
                                    ctypes.c_int64, ctypes.POINTER(MinimumFamilyC), ctypes.c_int64, _i64p,
                                    ctypes.POINTER(CollectStatsC)]
    L.bk_adjoint.argtypes = [c_ctx, ctypes.POINTER(AdjointParamsC), _dp, _dp, _dp, ctypes.POINTER(AdjointStatsC)]
    L.bk_fullspace_matvec.argtypes = [c_ctx, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_void_p,
                                      ctypes.c_void_p, ctypes.c_int]
    L.bk_fullspace_lanczos.argtypes = [c_ctx, ctypes.POINTER(LanczosParamsC), _dp, _dp,
                                       ctypes.POINTER(LanczosStatsC)]
    L.bk_sampler_run.argtypes = [c_ctx, ctypes.POINTER(SamplerConfigC), ctypes.c_uint64,
                                 ctypes.POINTER(SamplingResultC)]
    L.bk_sampling_result_release.argtypes = [ctypes.POINTER(SamplingResultC)]
    L.bk_sampling_result_release.restype = None
    L.bk_d_min.argtypes = [c_ctx, ctypes.c_int, ctypes.c_uint64, ctypes.c_int64, ctypes.c_int,
                           ctypes.POINTER(ctypes.c_int)]
    L.bk_random_states.argtypes = [ctypes.c_int, ctypes.c_uint64, ctypes.c_int64, _u64p]
    L.bk_steepest_descent.argtypes = [ctypes.c_int, _u64p, ctypes.c_int64, ctypes.c_uint64, _u64p, _i64p, _u64p]
    L.bk_select_trap.argtypes = [ctypes.c_int, ctypes.c_uint64, ctypes.c_int32, ctypes.c_double, _u64p, _i64p]
    _LIB = L
    return L


def _p(a, t):
    return a.ctypes.data_as(t) if a is not None else None


def labs_energy(n, states):
    L = load_library()
    s = np.ascontiguousarray(states, dtype=np.uint64).reshape(-1)
    out = np.empty(len(s), dtype=np.int64)
    st = L.bk_labs_energy(n, _p(s, _u64p), len(s), _p(out, _i64p))
    if st != BK_OK:
        raise BkError(st, "bk_labs_energy")
    return out


def random_states(n, seed, count):
    L = load_library()
    out = np.empty(count, dtype=np.uint64)
    st = L.bk_random_states(n, seed, count, _p(out, _u64p))
    if st != BK_OK:
        raise BkError(st, "bk_random_states")
    return out


def steepest_descent(n, starts, max_evals=0):
    """Returns (final_states, final_energies, evals) for each start (host, OpenMP)."""
    L = load_library()
    s = np.ascontiguousarray(starts, dtype=np.uint64).reshape(-1)
    fs = np.empty(len(s), dtype=np.uint64)
    fe = np.empty(len(s), dtype=np.int64)
    ev = np.empty(len(s), dtype=np.uint64)
    st = L.bk_steepest_descent(n, _p(s, _u64p), len(s), max_evals, _p(fs, _u64p), _p(fe, _i64p), _p(ev, _u64p))
    if st != BK_OK:
        raise BkError(st, "bk_steepest_descent")
    return fs, fe, ev


def select_trap(n, seed=42, n_descents=1000, quantile=0.05):
    """(bits, E0) of the benchmark trap policy (see include/bk_engine.h, bk_select_trap)."""
    L = load_library()
    b = ctypes.c_uint64()
    e = ctypes.c_int64()
    st = L.bk_select_trap(n, seed, n_descents, quantile, ctypes.byref(b), ctypes.byref(e))
    if st != BK_OK:
        raise BkError(st, "bk_select_trap")
    return int(b.value), int(e.value)


class Engine:
    """One bk_ctx: a device, a stream and the cached device buffers."""

    def __init__(self, device=0):
        self.L = load_library()
        self.device = device
        self.ctx = ctypes.c_void_p()
        st = self.L.bk_create(device, ctypes.byref(self.ctx))
        if st != BK_OK:
            raise BkError(st, self.L.bk_status_string(st).decode())

    def _check(self, st, what):
        if st != BK_OK:
            raise BkError(st, f"{what}: {self.L.bk_last_error(self.ctx).decode()}")

    def close(self):
        if self.ctx:
            self.L.bk_destroy(self.ctx)
            self.ctx = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def energy_table(self, n):
        out = np.empty(1 << n, dtype=np.uint16)
        self._check(self.L.bk_energy_table(self.ctx, n, _p(out, _u16p)), "bk_energy_table")
        return out

    def p_blind(self, n, e0):
        c = ctypes.c_uint64()
        p = ctypes.c_double()
        self._check(self.L.bk_p_blind(self.ctx, n, e0, ctypes.byref(c), ctypes.byref(p)), "bk_p_blind")
        return int(c.value), float(p.value)

    def evolve(self, n, s0, g, dt, n_steps, measure=None, e0=-1, precision=BK_C64, method=BK_FUSED,
               ordering=BK_ORDER_REFERENCE, diag_scale=0.0, norm_tol=0.0):
        """Returns (p_less, d_h, norm) at the flagged steps (measurement before stepping)."""
        flags = np.zeros(n_steps + 1, dtype=np.uint8)
        if measure is None:
            flags[:] = 1
        else:
            flags[np.asarray(list(measure), dtype=np.int64)] = 1
        g_arr = None
        gp = EvolveParams(n=n, precision=precision, method=method, ordering=ordering, s0=s0, e0=e0, dt=dt,
                          diag_scale=diag_scale, n_steps=n_steps, norm_tol=norm_tol)
        if np.ndim(g) == 0:
            gp.g_const = float(g)
        else:
            g_arr = np.ascontiguousarray(g, dtype=np.float64)
            if len(g_arr) != n_steps:
                raise ValueError("g schedule must have n_steps entries")
            gp.g = _p(g_arr, _dp)
        gp.measure = _p(flags, _u8p)
        m = int(flags.sum())
        p = np.zeros(m)
        d = np.zeros(m)
        nn = np.zeros(m)
        self._check(self.L.bk_evolve(self.ctx, ctypes.byref(gp), _p(p, _dp), _p(d, _dp), _p(nn, _dp)),
                    "bk_evolve")
        return p, d, nn

    def evolve_batch(self, instances, dt, n_steps, measure=None, precision=BK_C64, use_graph=True, lag=0,
                     diag_scale=0.0):
        """Many statevectors in one persistent launch.

        ``instances``: sequence of dicts with n, s0 and either g (scalar) or a per-step
        schedule; optional e0. Returns (p_less, d_h, norm) as [instance, measurement]."""
        flags = np.zeros(n_steps + 1, dtype=np.uint8)
        if measure is None:
            flags[:] = 1
        else:
            flags[np.asarray(list(measure), dtype=np.int64)] = 1
        arr = (BatchInstanceC * len(instances))()
        keep = []
        for i, d in enumerate(instances):
            arr[i].n = d["n"]
            arr[i].s0 = d["s0"]
            arr[i].e0 = d.get("e0", -1)
            g = d.get("g", 0.35)
            if np.ndim(g) == 0:
                arr[i].g_const = float(g)
            else:
                ga = np.ascontiguousarray(g, dtype=np.float64)
                keep.append(ga)
                arr[i].g = _p(ga, _dp)
        bp = BatchParamsC(precision=precision, n_steps=n_steps, dt=dt, diag_scale=diag_scale,
                          measure=_p(flags, _u8p), use_graph=1 if use_graph else 0, lag=lag)
        m = int(flags.sum())
        shape = (len(instances), m)
        p, d, nn = np.zeros(shape), np.zeros(shape), np.zeros(shape)
        self._check(self.L.bk_evolve_batch(self.ctx, ctypes.byref(bp), arr, len(instances), _p(p, _dp), _p(d, _dp),
                                           _p(nn, _dp)), "bk_evolve_batch")
        return p, d, nn

    def adjoint(self, n, s0, g_segments, dt, n_steps, segment_of_step=None, e0=-1, precision=BK_C64,
                objective=BK_OBJ_P_LESS, checkpoint_every=128, diag_scale=0.0, per_step=False):
        """O(T) and dO/dg_j of a piecewise-constant field schedule (adjoint method).

        Returns (value, grad[n_segments], stats dict); with ``per_step`` the stats
        also carry ``grad_steps`` (dO/dg_k for every step)."""
        g = np.ascontiguousarray(g_segments, dtype=np.float64)
        seg = None
        if segment_of_step is not None:
            seg = np.ascontiguousarray(segment_of_step, dtype=np.int32)
            if len(seg) != n_steps:
                raise ValueError("segment_of_step must have n_steps entries")
        ap = AdjointParamsC(n=n, precision=precision, s0=s0, e0=e0, dt=dt, diag_scale=diag_scale, n_steps=n_steps,
                            n_segments=len(g), g=_p(g, _dp),
                            segment_of_step=_p(seg, ctypes.POINTER(ctypes.c_int32)),
                            checkpoint_every=checkpoint_every, objective=objective)
        val = np.zeros(1)
        grad = np.zeros(len(g))
        gsteps = np.zeros(max(n_steps, 1)) if per_step else None
        st = AdjointStatsC()
        self._check(self.L.bk_adjoint(self.ctx, ctypes.byref(ap), _p(val, _dp), _p(grad, _dp), _p(gsteps, _dp),
                                      ctypes.byref(st)), "bk_adjoint")
        stats = {k: getattr(st, k) for k, _ in AdjointStatsC._fields_}
        if per_step:
            stats["grad_steps"] = gsteps[:n_steps]
        return float(val[0]), grad, stats

    def steepest_descent(self, n, starts, max_evals=0):
        """Device batched descent (bit-exact with the module-level host version):
        (final_states, final_energies, evals)."""
        st = np.ascontiguousarray(starts, dtype=np.uint64)
        fs = np.empty(len(st), dtype=np.uint64)
        fe = np.empty(len(st), dtype=np.int64)
        ev = np.empty(len(st), dtype=np.uint64)
        self._check(self.L.bk_steepest_descent_gpu(self.ctx, n, _p(st, _u64p), len(st), max_evals, _p(fs, _u64p),
                                                   _p(fe, _i64p), _p(ev, _u64p)), "bk_steepest_descent_gpu")
        return fs, fe, ev

    def collect_minima(self, n, seed=42, target_families=100, batch_size=4096, max_starts=100000):
        """Distinct local-minimum families (list of dicts, deepest first) and run statistics."""
        cap = int(target_families)
        arr = (MinimumFamilyC * cap)()
        cnt = ctypes.c_int64()
        st = CollectStatsC()
        self._check(self.L.bk_collect_minima(self.ctx, n, seed, target_families, batch_size, max_starts, arr, cap,
                                             ctypes.byref(cnt), ctypes.byref(st)), "bk_collect_minima")
        fams = [{k: getattr(arr[i], k) for k, _ in MinimumFamilyC._fields_} for i in range(min(cnt.value, cap))]
        return fams, {k: getattr(st, k) for k, _ in CollectStatsC._fields_}

    def d_min(self, n, bits, target=-1, max_d=-1):
        d = ctypes.c_int()
        self._check(self.L.bk_d_min(self.ctx, n, bits, target, max_d, ctypes.byref(d)), "bk_d_min")
        return int(d.value)

    def sampler_run(self, start_bits, precision=BK_C128, method=BK_FUSED, **cfg):
        """The reference's ISampler::sample(start_state, SamplerConfig) as a dict.

        ``cfg`` takes the SamplerConfig field names (sampler.cuh:235-260) with the
        reference's defaults."""
        defaults = dict(n=16, g=0.5, dt=0.05, t_max=60.0, num_sample_points=20, shots_per_point=100, seed=42,
                        num_sampling_seeds=3, seed_stride=10007, t_start=0.0, dt_sample=0.0, track_p_less=True,
                        verbose=True, record_trajectory=False, dt_trajectory=0.0)
        unknown = set(cfg) - set(defaults)
        if unknown:
            raise TypeError(f"unknown SamplerConfig fields: {sorted(unknown)}")
        defaults.update(cfg)
        c = SamplerConfigC(**{k: (int(v) if isinstance(v, bool) else v) for k, v in defaults.items()},
                           precision=precision, method=method)
        r = SamplingResultC()
        st = self.L.bk_sampler_run(self.ctx, ctypes.byref(c), start_bits, ctypes.byref(r))
        try:
            self._check(st, "bk_sampler_run")
            npt = r.n_points
            out = {k: getattr(r, k) for k, _ in SamplingResultC._fields_
                   if k not in ("unique_basis", "seed_stats", "time_points", "p_less_history", "dh_history")}
            out["time_points"] = np.ctypeslib.as_array(r.time_points, (npt,)).copy() if npt else np.zeros(0)
            out["p_less_history"] = np.ctypeslib.as_array(r.p_less_history, (npt,)).copy() if npt else np.zeros(0)
            out["dh_history"] = np.ctypeslib.as_array(r.dh_history, (npt,)).copy() if npt else np.zeros(0)
            nu = r.unique_basis_size
            out["unique_basis"] = np.ctypeslib.as_array(r.unique_basis, (nu,)).copy() if nu else np.zeros(0, np.uint64)
            out["seed_stats"] = [{k: getattr(r.seed_stats[i], k) for k, _ in SeedStatsC._fields_}
                                 for i in range(r.n_seed_stats)]
            return out
        finally:
            if st == BK_OK:
                self.L.bk_sampling_result_release(ctypes.byref(r))

    def fullspace_matvec(self, n, g, x, y, scale=None, method=BK_FUSED):
        """y = (scale E - g sum_j X_j) x on the device: x, y CUDA float64 tensors of 2^n
        elements on this engine's device (scale defaults to 1/n, the reference's
        normalize_by_n). method: BK_FUSED (tile passes) or BK_PLAIN (the reference's
        one-thread-per-state form). Returns after the product is complete."""
        import torch
        for t in (x, y):
            if not (t.is_cuda and t.dtype == torch.float64 and t.is_contiguous() and t.numel() == (1 << n)):
                raise ValueError("x and y must be contiguous CUDA float64 tensors of 2^n elements")
        torch.cuda.current_stream(x.device).synchronize()
        self._check(self.L.bk_fullspace_matvec(self.ctx, n, g, (1.0 / n) if scale is None else scale,
                                               ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(y.data_ptr()),
                                               int(method)),
                    "bk_fullspace_matvec")
        return y

    def fullspace_lanczos(self, n, g, num_eigenpairs=1, max_krylov_dim=100, tolerance=1e-12, normalize_by_n=True,
                          vectors=True):
        """The reference's Diagonalizer::solve_fullspace_lanczos (diagonalizer.cuh:377-560):
        (energies[num_eigenpairs], vectors [num_eigenpairs, 2^n] or None, info) with the
        tridiagonal matrix (alphas, betas) and the Krylov dimension reached in info."""
        alphas = np.zeros(max(max_krylov_dim, 1))
        betas = np.zeros(max(max_krylov_dim, 1))
        prm = LanczosParamsC(n=n, g=g, num_eigenpairs=num_eigenpairs, max_krylov_dim=max_krylov_dim,
                             tolerance=tolerance, normalize_by_n=int(bool(normalize_by_n)),
                             alphas=_p(alphas, _dp), betas=_p(betas, _dp))
        energies = np.zeros(num_eigenpairs)
        vec = np.zeros((num_eigenpairs, 1 << n)) if vectors else None
        st = LanczosStatsC()
        self._check(self.L.bk_fullspace_lanczos(self.ctx, ctypes.byref(prm), _p(energies, _dp),
                                                _p(vec, _dp) if vectors else None, ctypes.byref(st)),
                    "bk_fullspace_lanczos")
        m = st.krylov_dim
        info = {"krylov_dim": m, "matvecs": st.matvecs, "seconds": st.seconds, "alphas": alphas[:m].copy(),
                "betas": betas[:max(m - 1, 0)].copy()}
        return energies, vec, info

    def export_state(self, n):
        out = np.empty(2 << n)
        self._check(self.L.bk_export_state(self.ctx, _p(out, _dp)), "bk_export_state")
        return out[0::2] + 1j * out[1::2]

    def sample(self, randnums):
        r = np.ascontiguousarray(randnums, dtype=np.float64)
        out = np.empty(len(r), dtype=np.uint64)
        self._check(self.L.bk_sample(self.ctx, _p(r, _dp), len(r), _p(out, _u64p)), "bk_sample")
        return out

    OPTIONS = {"engine_mode": 0, "slab_lag": 1, "split_w2": 2, "e_source": 3, "a1_wide": 4, "adj_a1": 5,
               "wait_polls": 6, "test_hold_step": 7, "phase_table": 8}

    def set_option(self, name, value):
        self._check(self.L.bk_set_option(self.ctx, self.OPTIONS[name], int(value)), "bk_set_option")

    def get_option(self, name):
        v = ctypes.c_int64()
        self._check(self.L.bk_get_option(self.ctx, self.OPTIONS[name], ctypes.byref(v)), "bk_get_option")
        return int(v.value)

    def stream_handle(self):
        """The engine's cudaStream_t as an integer (for torch.cuda.ExternalStream)."""
        h = ctypes.c_void_p()
        self._check(self.L.bk_stream(self.ctx, ctypes.byref(h)), "bk_stream")
        return int(h.value or 0)

    def set_kernel_timing(self, enabled):
        self._check(self.L.bk_set_kernel_timing(self.ctx, 1 if enabled else 0), "bk_set_kernel_timing")

    def kernel_timing(self):
        out = {}
        i = 0
        while True:
            name = ctypes.c_char_p()
            launches = ctypes.c_int64()
            ms = ctypes.c_double()
            if self.L.bk_kernel_timing(self.ctx, i, ctypes.byref(name), ctypes.byref(launches),
                                       ctypes.byref(ms)) != BK_OK:
                break
            out[name.value.decode()] = (int(launches.value), float(ms.value))
            i += 1
        return out
