"""Pins the oracle's LABS energy core and trap generation to the reference.

Sources: data_raw/classical/exhaustive/{n}.csv and min_energies.csv (golden
tables), tests/test_labs_energy.cpp:8-117 and tests/test_d_min.cpp (known-answer
tests), tests/test_connector.cpp:270-279 (N=24 traps), and — when it was built in
this container — the reference's own compiled labs_energy.hpp / classical.cuh
(oracle/_ref).
"""
import random

import numpy as np
import pytest

from oracle import oracle as O


def test_energy_matches_exhaustive_tables(golden):
    g = golden("energy_exhaustive.json")
    for n_s, energies in g["full"].items():
        n = int(n_s)
        assert np.array_equal(O.energy_table(n).astype(np.int64), np.array(energies)), n
    for n_s, rows in g["sampled"].items():
        n = int(n_s)
        ck = np.zeros(n, dtype=np.int64)
        for row in rows:
            s, cks, e = row[0], row[1:-1], row[-1]
            O.lib().orc_labs_ck(n, s, ck.ctypes.data_as(O.i64p))
            assert list(ck[1:]) == cks
            assert O.labs_energy(n, s) == e


def test_known_answer_energies():
    # tests/test_labs_energy.cpp:10-21 — E(bits = N) for N = 2..10
    expected = [0, 0, 1, 1, 2, 6, 7, 35, 32, 24, 45]
    for n in range(2, 11):
        assert O.labs_energy(n, n) == expected[n]
    # tests/test_labs_energy.cpp:24-62 — Barker sequences
    assert O.labs_energy(5, 8) == 2
    assert O.labs_energy(7, (1 << 3) | (1 << 4) | (1 << 6)) == 3
    assert O.labs_energy(11, sum(1 << b for b in (3, 4, 5, 7, 8, 10))) == 5
    assert O.labs_energy(13, sum(1 << b for b in (5, 6, 9, 11))) == 6


def test_symmetry_invariance():
    # tests/test_labs_energy.cpp:91-117 — E is invariant under the order-8 group
    rng = random.Random(7)
    for n in range(4, 31):
        for _ in range(20):
            s = rng.randrange(1 << n)
            e = O.labs_energy(n, s)
            assert O.labs_energy(n, O.canonical(n, s)) == e
            assert O.labs_energy(n, (~s) & ((1 << n) - 1)) == e


def test_optimal_energies_and_counts(golden):
    # min_energies.csv columns: n, E*(n), lowest-index state with E = E*(n)
    for row in golden("min_energies.json"):
        n = row["n"]
        if n >= 3:
            assert O.lib().orc_known_optimal_energy(n) == row["energy"]
        assert O.labs_energy(n, row["first_state"]) == row["energy"]
        if 1 <= n <= 20:
            tab = O.energy_table(n)
            assert int(tab.min()) == row["energy"]
            assert int(np.nonzero(tab == row["energy"])[0][0]) == row["first_state"]


def _d_min_brute(n, s, target):
    tab = O.energy_table(n).astype(np.int64)
    below = np.nonzero(tab < target)[0]
    if len(below) == 0:
        return None
    return min(bin(int(x) ^ s).count("1") for x in below)


def test_d_min_brute_force():
    # tests/test_d_min.cpp — all states at N=6, sampled states at N=10
    for n, states in ((6, range(64)), (10, random.Random(3).sample(range(1024), 60))):
        for s in states:
            e = O.labs_energy(n, s)
            got = O.d_min(n, s, e)
            opt = O.lib().orc_known_optimal_energy(n)
            if e <= opt:
                assert got == n
            else:
                assert got == _d_min_brute(n, s, e)


def test_trap_tables(golden):
    t = golden("traps.json")
    # tests/test_connector.cpp:270-279 — N=24 exhaustive traps
    lv = {l["E0"]: l["orbits"] for l in t["orbits"]["24"]["levels"]}
    assert O.labs_energy(24, 0x5D2C6) == 44 and lv[44][0]["canonical_id"] == "0x5D2C6"
    assert O.labs_energy(24, 0x38C95) == 48 and lv[48][0]["canonical_id"] == "0x38C95"
    for n_s, d in t["orbits"].items():
        n = int(n_s)
        for level in d["levels"]:
            for o in level["orbits"][:3]:
                bits = int(o["canonical_id"], 16)
                assert O.labs_energy(n, bits) == level["E0"]
                assert int(o["bitstring"], 2) == bits
                if n <= 24:
                    assert O.d_min(n, bits, level["E0"]) == o["d_min"]
    for n_s, rows in t["results"].items():
        n = int(n_s)
        for r in rows[::3]:
            bits = int(r["trap_bits"], 16)
            assert O.labs_energy(n, bits) == int(r["trap_energy"])
            if n <= 20:
                assert O.d_min(n, bits, int(r["trap_energy"])) == int(r["d_min"])
                pb = O.count_below(n, int(r["trap_energy"])) / float(1 << n)
                assert pb == pytest.approx(float(r["p_blind"]), rel=6e-7, abs=1e-15)


@pytest.mark.skipif(O.ref_lib() is None, reason="reference tree was not present when the oracle was built")
def test_oracle_matches_reference_build():
    R = O.ref_lib()
    rng = random.Random(11)
    ck_a = np.zeros(64, dtype=np.int64)
    ck_b = np.zeros(64, dtype=np.int64)
    for n in range(2, 31):
        assert O.lib().orc_known_optimal_energy(n) == R.ref_known_optimal_energy(n)
        for _ in range(30):
            s = rng.randrange(1 << n)
            assert O.labs_energy(n, s) == R.ref_calc_energy(n, s)
            O.lib().orc_labs_ck(n, s, ck_a.ctypes.data_as(O.i64p))
            R.ref_calc_ck(n, s, ck_b.ctypes.data_as(O.i64p))
            assert list(ck_a[:n]) == list(ck_b[:n])
            assert O.canonical(n, s) == R.ref_canonical(n, s)
        for _ in range(3):
            s = rng.randrange(1 << n)
            if n <= 20:
                e = O.labs_energy(n, s)
                assert O.d_min(n, s, e) == R.ref_d_min(n, s, e, -1)
                assert O.d_min(n, s, e, 2) == R.ref_d_min(n, s, e, 2)
    for n, seed in ((12, 42), (24, 42), (28, 43), (30, 44)):
        a = O.random_states(n, seed, 200)
        b = np.zeros(200, dtype=np.uint64)
        R.ref_random_states(n, seed, 200, b.ctypes.data_as(O.u64p))
        assert np.array_equal(a, b)
        for s in a[:40]:
            assert O.steepest_descent(n, int(s)) == O.steepest_descent(n, int(s), use_ref=True)
            assert O.steepest_descent(n, int(s), 3 * n) == O.steepest_descent(n, int(s), 3 * n, use_ref=True)


def test_energy_levels_fit_the_full_phase_table():
    """The complex64 A1 kernels' full phase table (BK_OPT_PHASE_TABLE) indexes the
    level j = (E - c0) / 4 with c0 = floor(n/2) mod 4: C_k has the parity of n - k,
    an odd square is 1 mod 8 and an even one 0 mod 4, so every energy is c0 mod 4
    and at least c0. Checked on every state of n = 3..20 (the oracle's energy table,
    the restatement of labs_energy.hpp:121-149), and the table capacity compiled
    into the kernels (kPhaseTabMax) against the largest padded count, n = 30."""
    import os
    import re
    for n in range(3, 21):
        E = O.energy_table(n).astype(np.int64)
        c0 = (n // 2) & 3
        emax = (n - 1) * n * (2 * n - 1) // 6
        assert np.all(E % 4 == c0) and E.min() >= c0 and E.max() <= emax, n
    src = open(os.path.join(os.path.dirname(__file__), "..", "bernasconi-krylov_b200", "csrc",
                            "bk_persist.cuh")).read()
    cap = int(re.search(r"constexpr int kPhaseTabMax = (\d+);", src).group(1))
    for n in range(14, 31):
        emax = (n - 1) * n * (2 * n - 1) // 6
        n_j = (emax - ((n // 2) & 3)) // 4 + 1
        assert ((n_j + 1) & ~1) <= cap, n
