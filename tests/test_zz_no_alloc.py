"""bk_measure_noalloc: measurement of a caller-owned statevector for callers that
cannot let a library allocate device memory (a framework that owns all GPU memory
through its own allocator, or a loop that must not synchronise on an allocation).

The caller (here: torch) owns the statevector and the 3-double output; the entry
point's only scratch is a fixed array inside the library. Each case calls it twice
in a row and checks both results against the engine's regular measurement
(bk_evolve) of the same state, with the tolerances of the other parity tests:
complex128 1e-10 (1e-10 * n for <d_H>), complex64 1e-6 (3e-6 for <d_H>). bk_evolve
returns complex64 sums divided by the state's norm, so they are multiplied back by
the norm it reports before the comparison (this entry point returns raw sums). This file is
collected last so that a run stopping at the first failure has run every other test.
"""
import ctypes

import numpy as np
import pytest

import bk_b200 as bk

pytestmark = pytest.mark.gpu


def _lib():
    L = bk.load_library()
    L.bk_measure_noalloc.restype = ctypes.c_int
    L.bk_measure_noalloc.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_int64, ctypes.c_uint64,
                                     ctypes.c_void_p, ctypes.c_void_p]
    return L


@pytest.mark.parametrize("precision", [bk.BK_C128, bk.BK_C64])
@pytest.mark.parametrize("n", [16, 22])
def test_noalloc_matches_engine_measurement(precision, n):
    import torch
    bits, e0 = bk.select_trap(n, 42, 200, 0.05)
    steps = 24
    with bk.Engine(0) as eng:
        p, d, nn = eng.evolve(n, bits, 0.35, 0.05, steps, measure=[steps], e0=e0, precision=precision)
        state = eng.export_state(n)  # complex128 on the host, true scale
    dev = torch.device("cuda", 0)
    host = state if precision == bk.BK_C128 else state.astype(np.complex64)
    d_state = torch.view_as_real(torch.from_numpy(host)).contiguous().to(dev)
    d_out = torch.full((3,), float("nan"), dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    L = _lib()
    c128 = precision == bk.BK_C128
    tol, dtol = (1e-10, 1e-10 * n) if c128 else (1e-6, 3e-6)
    raw = 1.0 if c128 else nn[-1]  # complex64 results come back normalised
    for _ in range(2):  # two calls in a row share the library's scratch array
        d_out.fill_(float("nan"))
        st = L.bk_measure_noalloc(n, precision, d_state.data_ptr(), e0, bits, d_out.data_ptr(), stream.cuda_stream)
        assert st == 0, bk._lib.load_library().bk_status_string(st)
        stream.synchronize()
        got = d_out.cpu().numpy()
        assert abs(got[0] - p[-1] * raw) <= tol
        assert abs(got[1] - d[-1] * raw) <= dtol
        assert abs(got[2] - nn[-1]) <= tol


def test_noalloc_at_its_size_limit():
    """n = 30, the entry point's largest size (complex64, 8 GiB statevector): the
    same two-calls-in-a-row check against the engine's own measurement."""
    import psutil
    import torch
    if psutil.virtual_memory().available < 48 * 2**30:
        pytest.skip("needs ~40 GB of host memory for the exported n = 30 state")
    n, steps = 30, 2
    bits, e0 = bk.select_trap(n, 42, 100, 0.05)
    with bk.Engine(0) as eng:
        p, d, nn = eng.evolve(n, bits, 0.35, 0.05, steps, measure=[steps], e0=e0, precision=bk.BK_C64)
        state = eng.export_state(n).astype(np.complex64)
    dev = torch.device("cuda", 0)
    d_state = torch.view_as_real(torch.from_numpy(state)).to(dev)
    del state
    d_out = torch.full((3,), float("nan"), dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    L = _lib()
    for _ in range(2):
        d_out.fill_(float("nan"))
        st = L.bk_measure_noalloc(n, bk.BK_C64, d_state.data_ptr(), e0, bits, d_out.data_ptr(), stream.cuda_stream)
        assert st == 0
        stream.synchronize()
        got = d_out.cpu().numpy()
        assert abs(got[0] - p[-1] * nn[-1]) <= 1e-6
        assert abs(got[1] - d[-1] * nn[-1]) <= 3e-6
        assert abs(got[2] - nn[-1]) <= 1e-6


def test_noalloc_rejects_misaligned_pointers():
    L = _lib()
    # refused on the host before any device work (a float2 / double2 read off
    # its alignment would fault on the device)
    assert L.bk_measure_noalloc(16, bk.BK_C64, ctypes.c_void_p(4096 + 4), -1, 0, ctypes.c_void_p(4096), None) == 1
    assert L.bk_measure_noalloc(16, bk.BK_C128, ctypes.c_void_p(4096 + 8), -1, 0, ctypes.c_void_p(4096), None) == 1
    assert L.bk_measure_noalloc(16, bk.BK_C64, ctypes.c_void_p(4096), -1, 0, ctypes.c_void_p(4096 + 4), None) == 1


def test_noalloc_rejects_sizes_beyond_its_limit():
    L = _lib()
    # rejected on the host before any device work: n above the fixed limit of 30
    assert L.bk_measure_noalloc(31, bk.BK_C64, ctypes.c_void_p(16), -1, 0, ctypes.c_void_p(16), None) == 8
    assert L.bk_status_string(8).startswith(b"request beyond a fixed limit")
