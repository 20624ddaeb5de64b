"""The benchmarked configurations, pinned on the GPU with the knobs bench.py uses.

bench.py times N = 28 complex64 with the autotuner's cached choice for this
device (bk_b200/tuning/b200.json); these tests run that exact configuration
over the large configuration's full schedule and compare it with complex128 on
the same trap, schedule and step ordering (the reference's step psi <- M D psi,
src/sampling/sampler.cuh:604-618, and its reductions :149-195). complex128 is
itself pinned to the reference's own cuStateVec series at N = 24...30 by
tests/test_gpu_parity.py::test_golden_series_c128.

Bars (complex64 against complex128), written here:
  * |dP_<| <= C64_DP_BAR (1e-6) at every measured step;
  * |d<d_H>| <= C64_DH_BAR (1.2e-5) at every measured step (the reason is written
    beside the constants in tests/conftest.py);
  * state infidelity 1 - |<psi_64|psi_128>|^2 <= 1e-8 at the end of the run.
"""
import numpy as np
import pytest

import bk_b200 as bk
from bk_b200 import tune
from conftest import C64_DH_BAR, C64_DP_BAR

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def eng():
    e = bk.Engine(0)
    yield e
    e.close()


def _evolve_tuned(eng, n, precision, bits, e0, g, dt, steps, every):
    knobs = tune.apply(eng, n, precision)
    meas = list(range(0, steps + 1, every))
    try:
        return eng.evolve(n, bits, g, dt, steps, measure=meas, e0=e0, precision=precision), knobs
    finally:
        tune.apply_config(eng, tune.DEFAULTS)


def _infidelity(a, b):
    ov = np.vdot(a, b) / (np.linalg.norm(a) * np.linalg.norm(b))
    return 1.0 - abs(ov) ** 2


def test_headline_n28_c64_tuned_against_c128(eng):
    """N = 28, trap from the lowest 1% of 4000 seeded descents (seed 42), g =
    0.35, dt = 0.02, 2000 steps, P_< and <d_H> every 20 steps: bench.py's
    workload over the configuration's whole run, with the tuned knobs."""
    n, steps, every = 28, 2000, 20
    bits, e0 = bk.select_trap(n, 42, 4000, 0.01)
    (p64, d64, n64), knobs = _evolve_tuned(eng, n, bk.BK_C64, bits, e0, 0.35, 0.02, steps, every)
    assert knobs is not None, "no tuned entry for N = 28 complex64: bench.py would not run these knobs"
    s64 = eng.export_state(n)
    (p128, d128, n128), _ = _evolve_tuned(eng, n, bk.BK_C128, bits, e0, 0.35, 0.02, steps, every)
    s128 = eng.export_state(n)
    assert len(p64) == steps // every + 1
    assert np.max(np.abs(p64 - p128)) <= C64_DP_BAR
    assert np.max(np.abs(d64 - d128)) <= C64_DH_BAR
    assert np.max(np.abs(n128 - 1.0)) <= 1e-10
    assert _infidelity(s64, s128) <= 1e-8


def test_large_n30_c64_tuned_against_c128_and_golden(eng, golden):
    """N = 30 complex64 (8 GiB statevector, the reference's largest size,
    sampler.cuh:416-418) with its tuned knobs on the golden trap of
    data_processed/probability_dynamics_n30.csv (g = 0.35, dt = 0.05, 1200
    steps, every 10): against complex128 as above, and against the reference's
    cuStateVec series at its print precision plus the complex64 bar."""
    s = next(x for x in golden("series_n30.json")["series"] if abs(x["g"] - 0.35) < 1e-12)
    n, bits = 30, int(s["trap_bits"], 16)
    steps, every = int(round(s["t_max"] / s["dt"])), s["every"]
    (p64, d64, _), knobs = _evolve_tuned(eng, n, bk.BK_C64, bits, -1, s["g"], s["dt"], steps, every)
    assert knobs is not None
    (p128, d128, _), _ = _evolve_tuned(eng, n, bk.BK_C128, bits, -1, s["g"], s["dt"], steps, every)
    assert np.max(np.abs(p64 - p128)) <= C64_DP_BAR
    assert np.max(np.abs(d64 - d128)) <= C64_DH_BAR
    gp, gd = np.array(s["p_less"]), np.array(s["dh"])
    assert np.all(np.abs(p64 - gp) <= 6e-7 * np.abs(gp) + C64_DP_BAR)
    assert np.all(np.abs(d64 - gd) <= 5.01e-5 + C64_DH_BAR)
