"""Full phase table of the complex64 A1 kernels (BK_OPT_PHASE_TABLE).

The diagonal phase exp(-i dt/N E(s)) of the reference (src/sampling/sampler.cuh:73-91,
applied before the mixer at :604-618) is computed by the complex64 A1 kernels
either from a 16-entry level table with residual polynomials, or (phase_table = 1)
from one table entry per energy level, E = c0 + 4 j. Both are shear rotations of
the same angle rounded differently, so complex64 series stay within the complex64
bars of the oracle / complex128.
"""
import numpy as np
import pytest

import bk_b200 as bk
from bk_b200 import tune
from conftest import C64_DH_BAR, C64_DP_BAR
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def eng():
    e = bk.Engine(0)
    yield e
    tune.apply_config(e, tune.DEFAULTS)
    e.close()


def _run(eng, n, bits, e0, steps, every, precision, mode, a1, table, g=0.35, dt=0.02):
    tune.apply_config(eng, tune.DEFAULTS)
    eng.set_option("engine_mode", mode)
    eng.set_option("slab_lag", 2)
    eng.set_option("a1_wide", a1)
    eng.set_option("phase_table", table)
    try:
        return eng.evolve(n, bits, g, dt, steps, measure=list(range(0, steps + 1, every)), e0=e0,
                          precision=precision)
    finally:
        tune.apply_config(eng, tune.DEFAULTS)


@pytest.mark.parametrize("mode", [1, 2])
@pytest.mark.parametrize("a1", [0, 1, 2, 3])
def test_phase_table_matches_oracle(eng, mode, a1):
    """complex64 with the full table, every A1 kernel that takes it, both
    per-pass schedules: within the complex64 bars of the complex128 oracle."""
    n, steps = 22, 40
    bits, e0 = bk.select_trap(n, 6, 200, 0.05)
    p, d, _ = _run(eng, n, bits, e0, steps, 5, bk.BK_C64, mode, a1, 1)
    po, do, _ = O.trotter_evolve(n, bits, e0, 0.35, 0.02, steps, measure=list(range(0, steps + 1, 5)))
    assert np.max(np.abs(p - po)) <= C64_DP_BAR
    assert np.max(np.abs(d - do)) <= C64_DH_BAR


def test_phase_table_long_run_against_c128(eng):
    """The N = 24 configuration's length (1000 steps, every 10) with the table on
    the 512-thread A1 and the fused strided pass, against complex128."""
    n, steps = 24, 1000
    bits, e0 = bk.select_trap(n, 42, 1000, 0.05)
    p64, d64, _ = _run(eng, n, bits, e0, steps, 10, bk.BK_C64, 2, 1, 1)
    p128, d128, _ = _run(eng, n, bits, e0, steps, 10, bk.BK_C128, 1, 0, 0)
    assert np.max(np.abs(p64 - p128)) <= C64_DP_BAR
    assert np.max(np.abs(d64 - d128)) <= C64_DH_BAR


def test_phase_table_ignored_where_unused(eng):
    """complex128 and the persistent schedule (mode 0) do not take the table:
    their series are bit-identical with the option on and off."""
    for n, prec, a1, mode in ((21, bk.BK_C128, 1, 1), (22, bk.BK_C64, 0, 0)):
        bits, e0 = bk.select_trap(n, 6, 200, 0.05)
        off = _run(eng, n, bits, e0, 12, 3, prec, mode, a1, 0)
        on = _run(eng, n, bits, e0, 12, 3, prec, mode, a1, 1)
        for a, b in zip(off, on):
            assert np.array_equal(a, b), (n, prec)
