"""CPU checks of the tile engine's round plans, read from the CUDA headers.

A 64 KB tile holds 4096 16-byte elements; a round assigns its 12 tile bits to
register, lane and warp bits (`Plan<double>`, `StridedR2`, `PlanA1Wide`,
`PlanA1Warp` in csrc/bk_fused.cuh and csrc/bk_persist.cuh). Checked here:
every round covers the tile exactly once; every 16-byte shared-memory access is
bank-conflict free under the layout it reads (the TMA's linear or 128-byte
swizzled stage, or the engine's XOR swizzle); and the narrowest barrier each
transition between rounds needs — none (the same thread on both sides of every
slot), a warp (`__syncwarp`), a warp pair (named barrier) or the CTA — which the
kernels' barriers must match or exceed."""
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "bernasconi-krylov_b200", "csrc")


def _consts(struct, fname):
    """uint32 constants of a plan struct, e.g. {'R1_REG': 0x47, ...}."""
    src = open(os.path.join(CSRC, fname)).read()
    m = re.search(r"struct " + re.escape(struct) + r"\s*(?:\{|:)(.*?)\n\};", src, re.S)
    assert m, struct
    return {k: int(v, 16) for k, v in re.findall(r"(\w+)\s*=\s*(0x[0-9A-Fa-f]+)", m.group(1))}


def pdep(x, mask):
    r, b = 0, 0
    for i in range(12):
        if mask >> i & 1:
            if x >> b & 1:
                r |= 1 << i
            b += 1
    return r


def swz(i):  # the engine's XOR swizzle (swz<double> in csrc/bk_fused.cuh)
    return i ^ (((i >> 3) ^ (i >> 6) ^ (i >> 9)) & 7)


def tma128(e):  # the 128-byte TMA swizzle in 16-byte elements: chunk bits 0-2 ^= row bits
    return e ^ ((e >> 3) & 7)


def linear(e):
    return e


def owners(nthr, reg, lane, warp):
    """element -> thread for one round."""
    out = {}
    nreg = bin(reg).count("1")
    for tid in range(nthr):
        b = pdep(tid & 31, lane) | pdep(tid >> 5, warp)
        for j in range(1 << nreg):
            e = b | pdep(j, reg)
            assert e not in out, "element held twice"
            out[e] = tid
    assert sorted(out) == list(range(4096)), "round does not cover the tile"
    return out


def conflict_free(nthr, reg, lane, warp, layout):
    """Every 128-bit access: each quarter warp hits 8 distinct 16-byte bank groups."""
    nreg = bin(reg).count("1")
    for w in range(nthr // 32):
        for j in range(1 << nreg):
            for q in range(4):
                groups = {layout(pdep(w * 32 + q * 8 + l & 31, lane) | pdep(w, warp) | pdep(j, reg)) & 7
                          for l in range(8)}
                if len(groups) != 8:
                    return False
    return True


def barrier_width(a, b):
    """Smallest group holding both threads of every slot touched on either side."""
    pairs = [(a[s], b[s]) for s in a]
    if all(x == y for x, y in pairs):
        return "none"
    if all(x >> 5 == y >> 5 for x, y in pairs):
        return "warp"
    if all(x >> 6 == y >> 6 for x, y in pairs):
        return "pair"
    return "cta"


def slots(own, layout):
    return {layout(e): t for e, t in own.items()}


def rounds_check(nthr, rounds, first_layout):
    """rounds: [(REG, LANE, WARP)]; round 1 reads `first_layout`, every later round
    reads the XOR swizzle; each round but the last stores back swizzled in its own
    layout. Returns the barrier widths needed between consecutive accesses."""
    widths = []
    prev = None
    for i, (reg, lane, warp) in enumerate(rounds):
        own = owners(nthr, reg, lane, warp)
        read_layout = first_layout if i == 0 else swz
        assert conflict_free(nthr, reg, lane, warp, read_layout), f"round {i + 1} read conflicts"
        rd = slots(own, read_layout)
        if prev is not None:
            widths.append(barrier_width(prev, rd))
        if i + 1 < len(rounds):
            assert conflict_free(nthr, reg, lane, warp, swz), f"round {i + 1} store conflicts"
            st = slots(own, swz)
            widths.append(barrier_width(rd, st))
            prev = st
    return widths


def test_a1_256_thread_plan():
    P = _consts("Plan<double>", "bk_fused.cuh")
    w = rounds_check(256, [(P["A1_R1_REG"], P["A1_R1_LANE"], P["A1_R1_WARP"]),
                           (P["A1_R2_REG"], P["A1_R2_LANE"], P["A1_R2_WARP"]),
                           (P["A1_R3_REG"], P["A1_R3_LANE"], P["A1_R3_WARP"])], linear)
    # process_a1: warp_sync, warp_sync, (in-place store), CTA barrier
    assert w == ["warp", "warp", "none", "cta"]
    assert P["A1_R1_REG"] | P["A1_R2_REG"] | P["A1_R3_ACT"] == 0xFFF


def test_a1_512_thread_plan():
    P = _consts("PlanA1Wide", "bk_persist.cuh")
    w = rounds_check(512, [(P[f"R{k}_REG"], P[f"R{k}_LANE"], P[f"R{k}_WARP"]) for k in (1, 2, 3, 4)], linear)
    # a1_wide_tile: warp_sync, warp_sync, (in place), pair_sync, (in place), CTA barrier
    assert w == ["warp", "warp", "none", "pair", "none", "cta"]
    assert P["R1_REG"] | P["R2_REG"] | P["R3_REG"] | P["R4_REG"] == 0xFFF


def test_a1_warp_local_plan():
    P = _consts("PlanA1Warp", "bk_persist.cuh")
    w = rounds_check(256, [(P["R1_REG"], P["R1_LANE"], P["WARP"]), (P["R2_REG"], P["R2_LANE"], P["WARP"])], tma128)
    # round 1's swizzled store lands in the slots the same thread read (both swizzles only permute
    # element bits 0-2, which are round-1 register bits), so no barrier is needed there (the kernels'
    # warp_sync is stronger than required); round 1 -> 2 stays inside the warp; no CTA barrier
    assert w == ["none", "warp"]
    assert P["WARP"] == 0xE00  # each warp owns the 512 elements with its warp bits 9-11
    # element bits 0-8: rounds 1 and 2 plus bit 8 across lanes 16 apart (round-2 lane bit 4)
    assert P["R1_REG"] | P["R2_REG"] | pdep(16, P["R2_LANE"]) == 0x1FF
    # 128-byte runs in the global stores: round-2 lanes 0-7 are element bits 0-2
    assert all(pdep(l, P["R2_LANE"]) == l for l in range(8))


@pytest.mark.parametrize("W", [5, 6, 7, 8, 9])
def test_strided_plans(W):
    P = _consts("Plan<double>", "bk_fused.cuh")
    cp = 12 - W
    r2 = {"REG": 0xF0 if W <= 8 else 0x78, "LANE": 0x10F if W <= 8 else 0x187, "WARP": 0xE00}
    src = open(os.path.join(CSRC, "bk_fused.cuh")).read()
    assert "(W <= 8) ? 0xF0u : 0x78u" in src and "(W <= 8) ? 0x10Fu : 0x187u" in src  # StridedR2 as restated
    w = rounds_check(256, [(P["S_R1_REG"], P["S_R1_LANE"], P["S_R1_WARP"]), (r2["REG"], r2["LANE"], r2["WARP"])],
                     linear)
    # process_s: warp_sync before the swizzled store, CTA barrier after it
    assert w == ["warp", "cta"]
    act = ((1 << W) - 1) << cp
    covered = (P["S_R1_REG"] & act) | (r2["REG"] & act) | (1 << 7 if W == 9 else 0)
    assert covered == act  # every active (high) tile bit is butterflied once; W = 9 adds the lane-shuffle bit 7
    assert cp >= 3  # every global access is a run of >= 8 elements (128 bytes)
