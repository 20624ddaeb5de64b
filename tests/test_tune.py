"""CPU checks of the autotuner's search space and cache (no device needed)."""
import json

import bk_b200 as bk
from bk_b200 import tune


def test_candidates_cover_modes_lags_and_valid_splits():
    c = tune.candidates(28, bk.BK_C64)  # 27 element bits: A1 12 + 15 strided, default S2 width 8
    assert {x["engine_mode"] for x in c} == {0, 1, 2, 3}
    assert {x.get("phase_table", 0) for x in c if x["engine_mode"] in (1, 2, 3)} == {0, 1}
    assert {x["split_w2"] for x in c} == {0, 7, 9}
    assert {x["slab_lag"] for x in c if x["engine_mode"] == 0} == {1, 2, 3, 4, 6}
    assert {x["slab_lag"] for x in c if x["engine_mode"] == 2} == {1, 2, 3}
    assert {x["e_source"] for x in c} == {0, 1}
    assert {x["a1_wide"] for x in c if x["engine_mode"] == 1} == {0, 1, 2, 3}
    assert {x["a1_wide"] for x in c if x["engine_mode"] == 2} == {0, 1, 2, 3}
    for n, prec in ((30, bk.BK_C64), (30, bk.BK_C128), (22, bk.BK_C64), (14, bk.BK_C64)):
        np_ = n - 1 if prec == bk.BK_C64 else n
        for x in tune.candidates(n, prec):
            # the warp-local A1 leaves np - 9 bits to the strided passes, S2 at least 3
            rest = np_ - (9 if x["a1_wide"] in (2, 3) else tune.ELEM_BITS)
            w = x["split_w2"] or tune.default_w2(rest)
            assert 1 <= w <= 9 and w <= rest and rest - w <= 9
            assert x["a1_wide"] not in (2, 3) or (w >= 3 and x["engine_mode"] in (1, 2, 3) and rest <= 18)
            # the fused strided pass is only tried where a third pass is left to fuse
            assert x["engine_mode"] not in (2, 3) or rest - w >= 1
            # the full phase table: complex64 per-pass schedules only
            assert not x.get("phase_table") or (prec == bk.BK_C64 and x["engine_mode"] in (1, 2, 3))


def test_cache_round_trip(tmp_path):
    p = str(tmp_path / "t.json")
    cache = {"dev/148sm": {"c64/n28": {"best": {"engine_mode": 1, "slab_lag": 3, "split_w2": 0}}}}
    tune.save_cache(cache, p)
    assert tune.load_cache(p) == cache
    assert json.load(open(p))["dev/148sm"]["c64/n28"]["best"]["engine_mode"] == 1
    assert tune.entry_key(28, bk.BK_C64) == "c64/n28"
    assert tune.batch_key([{"n": 16}, {"n": 22}, {"n": 16}], bk.BK_C64) == "batch/c64/3x16-22"


def test_committed_cache_is_well_formed():
    cache = tune.load_cache()
    for dev, entries in cache.items():
        for key, e in entries.items():
            assert "best" in e and e["amp_steps_per_s"] > 0
            if not key.startswith("batch/"):
                assert set(e["best"]) <= set(tune.KNOBS)
