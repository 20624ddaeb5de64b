"""Batched evolution (bk_evolve_batch): many statevectors of uneven n in one
persistent launch, optionally through a captured CUDA graph. Each instance must
reproduce its own single-statevector run of the same engine bit for bit (same tile
arithmetic, same fixed-order reductions), and the complex128 oracle to 1e-10."""
import numpy as np
import pytest

import bk_b200 as bk
from conftest import C64_DH_BAR, C64_DP_BAR
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def eng():
    e = bk.Engine(0)
    yield e
    e.close()


def _instances(ns, seed):
    rng = np.random.default_rng(seed)
    out = []
    for j, n in enumerate(ns):
        bits, e0 = bk.select_trap(n, 42 + j, 200, 0.05)
        out.append(dict(n=n, s0=bits, e0=e0, g=float(rng.uniform(0.2, 0.5))))
    return out


@pytest.mark.parametrize("precision", [bk.BK_C64, bk.BK_C128])
def test_batch_equals_single_runs(eng, precision):
    ns = [16, 14, 18, 20, 16, 22, 15, 19] if precision == bk.BK_C64 else [13, 16, 18, 20, 14, 21]
    inst = _instances(ns, 1)
    steps = 30
    meas = list(range(0, steps + 1, 3))
    eng.set_option("engine_mode", 0)
    pb, db, nb = eng.evolve_batch(inst, 0.02, steps, measure=meas, precision=precision, use_graph=True)
    pg, dg, _ = eng.evolve_batch(inst, 0.02, steps, measure=meas, precision=precision, use_graph=False)
    assert np.array_equal(pb, pg) and np.array_equal(db, dg)
    for i, d in enumerate(inst):
        p, dd, nn = eng.evolve(d["n"], d["s0"], d["g"], 0.02, steps, measure=meas, e0=d["e0"], precision=precision)
        assert np.array_equal(pb[i], p) and np.array_equal(db[i], dd) and np.array_equal(nb[i], nn), i


def test_batch_matches_oracle_c128(eng):
    inst = _instances([13, 15, 17], 2)
    steps = 20
    pb, db, _ = eng.evolve_batch(inst, 0.05, steps, precision=bk.BK_C128)
    for i, d in enumerate(inst):
        po, do, _ = O.trotter_evolve(d["n"], d["s0"], d["e0"], d["g"], 0.05, steps)
        assert np.max(np.abs(pb[i] - po)) <= 1e-10
        assert np.max(np.abs(db[i] - do)) <= 1e-10 * d["n"]


def test_batch_piecewise_schedules_c64(eng):
    rng = np.random.default_rng(3)
    steps = 24
    inst = []
    for j, n in enumerate([16, 18, 14]):
        bits, e0 = bk.select_trap(n, 7 + j, 200, 0.05)
        inst.append(dict(n=n, s0=bits, e0=e0, g=rng.uniform(0.25, 0.45, size=steps)))
    pb, db, nb = eng.evolve_batch(inst, 0.02, steps, precision=bk.BK_C64)
    for i, d in enumerate(inst):
        po, do, _ = O.trotter_evolve(d["n"], d["s0"], d["e0"], d["g"], 0.02, steps)
        assert np.max(np.abs(pb[i] - po)) <= C64_DP_BAR
        assert np.max(np.abs(db[i] - do)) <= C64_DH_BAR
        assert np.max(np.abs(nb[i] - 1.0)) <= 1e-5


def test_batch_rejects_small_n(eng):
    with pytest.raises(bk.BkError) as e:
        eng.evolve_batch([dict(n=10, s0=3, g=0.3)], 0.02, 4, precision=bk.BK_C64)
    assert e.value.status == bk._lib.BK_ERR_UNSUPPORTED
