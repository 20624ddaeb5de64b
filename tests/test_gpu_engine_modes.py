"""The two schedules of the tile engine — the persistent dataflow kernel and one
grid launch per pass — run the same tile arithmetic and the same fixed-order
reductions, so their measured series must agree bit for bit (and the complex128
series with the oracle to 1e-10)."""
import numpy as np
import pytest

import bk_b200 as bk
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def eng():
    e = bk.Engine(0)
    yield e
    e.set_option("engine_mode", 0)
    e.close()


@pytest.mark.parametrize("n,precision", [(16, bk.BK_C64), (22, bk.BK_C64), (24, bk.BK_C64), (15, bk.BK_C128),
                                         (21, bk.BK_C128), (23, bk.BK_C128)])
def test_grid_mode_equals_persistent(eng, n, precision):
    bits, e0 = bk.select_trap(n, 11, 200, 0.05)
    steps = 30
    meas = list(range(0, steps + 1, 5))
    g = np.random.default_rng(n).uniform(0.25, 0.45, steps)
    out = []
    for mode in (0, 1):
        eng.set_option("engine_mode", mode)
        out.append(eng.evolve(n, bits, g, 0.02, steps, measure=meas, e0=e0, precision=precision))
    eng.set_option("engine_mode", 0)
    for a, b in zip(out[0], out[1]):
        assert np.array_equal(a, b)


def test_grid_mode_matches_oracle_c128(eng):
    n, steps = 17, 24
    bits, e0 = bk.select_trap(n, 5, 200, 0.05)
    eng.set_option("engine_mode", 1)
    p, d, nn = eng.evolve(n, bits, 0.35, 0.05, steps, e0=e0, precision=bk.BK_C128)
    eng.set_option("engine_mode", 0)
    po, do, no = O.trotter_evolve(n, bits, e0, 0.35, 0.05, steps)
    assert np.max(np.abs(p - po)) <= 1e-10
    assert np.max(np.abs(d - do)) <= 1e-10 * n
    assert np.max(np.abs(nn - 1.0)) <= 1e-10
