"""Failure paths of the engine, exercised without faulting the GPU.

The reference reports CUDA failures by throwing std::runtime_error from its
CHECK_CUDA / CHECK_CUSTATEVEC macros (src/sampling/sampler.cuh:31-47); the C ABI
returns a status instead and the context must stay usable afterwards.

* BK_ERR_NORM: a norm tolerance tighter than complex64 rounding allows.
* BK_ERR_TIMEOUT: the persistent engine's test hook makes one step's dependency
  unreachable (a completion that no task will ever signal), so the bounded
  dependency wait runs out, every CTA leaves, and the host reads the status. No
  wait is unbounded, nothing traps, no memory is touched out of bounds.
"""
import numpy as np
import pytest

import bk_b200 as bk
from conftest import C64_DH_BAR, C64_DP_BAR
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _trap(n, seed=3):
    start = int(O.random_states(n, seed, 1)[0])
    bits, e0, _, _ = O.steepest_descent(n, start)
    return bits, e0


def test_norm_tolerance_reports_bk_err_norm():
    n, steps = 20, 12
    bits, e0 = _trap(n)
    with bk.Engine(0) as eng:
        with pytest.raises(bk.BkError) as e:
            eng.evolve(n, bits, 0.35, 0.05, steps, e0=e0, precision=bk.BK_C64, norm_tol=1e-12)
        assert e.value.status == bk._lib.BK_ERR_NORM
        # complex128 keeps its norm to ~1e-14: the same schedule passes a 1e-10 band
        p, d, nn = eng.evolve(n, bits, 0.35, 0.05, steps, e0=e0, precision=bk.BK_C128, norm_tol=1e-10)
        assert np.max(np.abs(nn - 1.0)) <= 1e-10
        # the context is usable after the failure and its results are right
        po, do, _ = O.trotter_evolve(n, bits, e0, 0.35, 0.05, steps)
        p64, d64, _ = eng.evolve(n, bits, 0.35, 0.05, steps, e0=e0, precision=bk.BK_C64)
        assert np.max(np.abs(p64 - po)) <= C64_DP_BAR


@pytest.mark.parametrize("precision", [bk.BK_C64, bk.BK_C128])
def test_lost_dependency_reports_bk_err_timeout(precision):
    n, steps = 20, 4
    bits, e0 = _trap(n, 5)
    with bk.Engine(0) as eng:
        eng.set_option("engine_mode", 0)
        eng.set_option("wait_polls", 2000)
        eng.set_option("test_hold_step", 1)
        with pytest.raises(bk.BkError) as e:
            eng.evolve(n, bits, 0.35, 0.05, steps, e0=e0, precision=precision)
        assert e.value.status == bk._lib.BK_ERR_TIMEOUT
        assert "bounded device wait" in str(e.value)
        # hook off: the same context runs the same schedule to the oracle's results
        eng.set_option("test_hold_step", -1)
        eng.set_option("wait_polls", 0)
        po, do, _ = O.trotter_evolve(n, bits, e0, 0.35, 0.05, steps)
        p, d, _ = eng.evolve(n, bits, 0.35, 0.05, steps, e0=e0, precision=precision)
        c64 = precision == bk.BK_C64
        assert np.max(np.abs(p - po)) <= (C64_DP_BAR if c64 else 1e-10)
        assert np.max(np.abs(d - do)) <= (C64_DH_BAR if c64 else 1e-10 * n)


def test_option_ranges_are_checked():
    with bk.Engine(0) as eng:
        for name, bad in (("wait_polls", 10), ("wait_polls", 1 << 30), ("test_hold_step", -2)):
            with pytest.raises(bk.BkError) as e:
                eng.set_option(name, bad)
            assert e.value.status == bk._lib.BK_ERR_INVALID
        assert eng.get_option("test_hold_step") == -1
        assert eng.get_option("wait_polls") == 0
