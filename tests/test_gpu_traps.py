"""Trap generation on the device: the warp-per-start steepest descent is
bit-exact (final state, energy, evaluation count) with the host descent and with
the reference's own ClassicalOptimizer::steepest_descent compiled from its
sources (oracle/_ref), and the minima collector reproduces a CPU restatement of
collect_distinct_minima_gpu (classical.cuh:861-959) family by family."""
import numpy as np
import pytest

import bk_b200 as bk
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def eng():
    e = bk.Engine(0)
    yield e
    e.close()


@pytest.mark.parametrize("n", [3, 5, 12, 20, 28, 31, 32, 33, 40, 63])
def test_device_descent_bit_exact(eng, n):
    starts = bk.random_states(n, 100 + n, 777)
    for budget in (0, 3 * n + 1):
        fs, fe, ev = eng.steepest_descent(n, starts, budget)
        hs, he, hv = bk.steepest_descent(n, starts, budget)
        assert np.array_equal(fs, hs) and np.array_equal(fe, he) and np.array_equal(ev, hv)
        if n <= 32:
            for j in range(0, 777, 97):
                r = O.steepest_descent(n, int(starts[j]), max_evals=budget, use_ref=True)
                assert (int(fs[j]), int(fe[j]), int(ev[j])) == r[:3]


def _cpu_collect(n, seed, target, batch, max_starts):
    rng_states = bk.random_states(n, seed, max_starts)
    fams, order, total_evals, starts, stagnant = {}, [], 0, 0, 0
    while len(fams) < target and starts < max_starts:
        st = rng_states[starts:starts + batch]
        fs, fe, ev = bk.steepest_descent(n, st, 0)
        starts += batch
        fresh = 0
        for i in range(batch):
            total_evals += int(ev[i])
            c = O.canonical(n, int(fs[i]))
            if c not in fams:
                fams[c] = dict(canonical_state=c, sample_state=int(fs[i]), energy=int(fe[i]), times_visited=1,
                               evals_to_first_find=total_evals)
                order.append(c)
                fresh += 1
                if len(fams) >= target:
                    break
            else:
                fams[c]["times_visited"] += 1
        stagnant = 0 if fresh else stagnant + 1
        if stagnant >= 4:
            break
    out = [fams[c] for c in order]
    out.sort(key=lambda f: (f["energy"], -f["times_visited"]))  # stable: discovery order breaks ties
    return out


@pytest.mark.parametrize("n,target", [(14, 40), (18, 1000)])
def test_collect_minima_matches_cpu_restatement(eng, n, target):
    fams, st = eng.collect_minima(n, seed=7, target_families=target, batch_size=256, max_starts=20000)
    ref = _cpu_collect(n, 7, target, 256, 20000)
    assert len(fams) == len(ref)
    for i, (a, b) in enumerate(zip(fams, ref)):
        assert a["id"] == i + 1
        for k in b:
            assert a[k] == b[k], (i, k)
    assert st["total_starts"] % 256 == 0
    assert [f["energy"] for f in fams] == sorted(f["energy"] for f in fams)
