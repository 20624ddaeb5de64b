"""CPU checks of the C ABI: the library builds/loads, exports every symbol that
include/bk_engine.h declares, rejects bad input on the host, and refuses to run
without a CUDA device (no silent CPU fallback)."""
import ctypes
import os
import re

import numpy as np
import pytest

import bk_b200 as bk
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    syms = set()
    for name in os.listdir(os.path.join(ROOT, "include")):
        if name.endswith(".h"):
            text = open(os.path.join(ROOT, "include", name)).read()
            text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
            syms |= set(re.findall(r"\b(bk_[a-z0-9_]+)\s*\(", text))
    return sorted(syms)


def test_library_exports_every_declared_symbol():
    L = bk.load_library()
    syms = declared_symbols()
    assert len(syms) >= 10
    for s in syms:
        assert hasattr(L, s), s
    assert L.bk_abi_version() == 1


def test_host_energy_matches_oracle():
    rng = np.random.default_rng(5)
    for n in (5, 12, 20, 28, 30):
        s = rng.integers(0, 1 << n, size=200, dtype=np.uint64)
        got = bk.labs_energy(n, s)
        assert [O.labs_energy(n, int(x)) for x in s] == list(got)


def test_host_argument_checks():
    L = bk.load_library()
    out = np.zeros(1, dtype=np.int64)
    s = np.zeros(1, dtype=np.uint64)
    assert L.bk_labs_energy(0, s.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)), 1,
                            out.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))) == bk._lib.BK_ERR_INVALID
    assert L.bk_create(0, None) == bk._lib.BK_ERR_INVALID
    assert L.bk_evolve(None, None, None, None, None) == bk._lib.BK_ERR_INVALID
    assert L.bk_status_string(bk._lib.BK_ERR_TIMEOUT) == b"device-side wait timed out"


@pytest.mark.skipif(os.environ.get("CUDA_VISIBLE_DEVICES") is None and os.path.exists("/dev/nvidia0"),
                    reason="a GPU is present")
def test_no_device_is_an_error_not_a_fallback():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(bk.BkError) as e:
        bk.Engine(0)
    assert e.value.status == bk._lib.BK_ERR_NO_DEVICE


def test_trap_generation_matches_reference_code():
    # random starts and descents are bit-exact with the reference's ClassicalOptimizer
    # (restated in the oracle, itself pinned to the reference's compiled code)
    for n, seed in ((12, 42), (24, 42), (28, 43)):
        starts = bk.random_states(n, seed, 300)
        assert np.array_equal(starts, O.random_states(n, seed, 300))
        fs, fe, ev = bk.steepest_descent(n, starts)
        for i in range(0, 300, 7):
            ofs, ofe, oev, _ = O.steepest_descent(n, int(starts[i]))
            assert (int(fs[i]), int(fe[i]), int(ev[i])) == (ofs, ofe, oev)
        fs2, fe2, ev2 = bk.steepest_descent(n, starts[:20], max_evals=3 * n)
        for i in range(20):
            assert (int(fs2[i]), int(fe2[i]), int(ev2[i])) == O.steepest_descent(n, int(starts[i]), 3 * n)[:3]


def test_select_trap_policy():
    n, seed, k, q = 16, 42, 200, 0.05
    bits, e0 = bk.select_trap(n, seed, k, q)
    starts = O.random_states(n, seed, k)
    res = [O.steepest_descent(n, int(s))[:2] for s in starts]
    opt = O.lib().orc_known_optimal_energy(n)
    kept = sorted(e for _, e in res if e > opt)
    thr = kept[int(np.floor(q * (len(kept) - 1)))]
    first = next((b, e) for b, e in res if opt < e <= thr)
    assert (bits, e0) == first
    assert O.labs_energy(n, bits) == e0 and e0 > opt


def test_oracle_trap_selection_equals_library():
    # bench.py's reference arm selects its trap with the oracle (never the
    # product library): both must give the same trap for every benchmark size
    for n, seed, k, q in ((16, 42, 200, 0.05), (24, 42, 1000, 0.05), (28, 42, 4000, 0.01), (30, 42, 4000, 0.01)):
        assert O.select_trap(n, seed, k, q) == tuple(bk.select_trap(n, seed, k, q))
        assert O.select_trap(n, seed, k, q, use_ref=False) == tuple(bk.select_trap(n, seed, k, q))
