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
                ("measure", _u8p), ("norm_tol", ctypes.c_double)]


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

    def export_state(self, n):
        out = np.empty(2 << n)
        self._check(self.L.bk_export_state(self.ctx, _p(out, _dp)), "bk_export_state")
        return out[0::2] + 1j * out[1::2]

    def sample(self, randnums):
        r = np.ascontiguousarray(randnums, dtype=np.float64)
        out = np.empty(len(r), dtype=np.uint64)
        self._check(self.L.bk_sample(self.ctx, _p(r, _dp), len(r), _p(out, _u64p)), "bk_sample")
        return out

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
