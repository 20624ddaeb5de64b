"""CPU model checks of the fused strided pass's task protocol (csrc/bk_s23.cuh).

The kernels decode a task from its claim index in closed form (s23_decode); the
host builds the same order explicitly (S3 tiles of slab h, then the S2 tiles of
slab h - lag) and checks the two agree on the first run of a geometry. Here the
closed form is restated and compared with that order for many geometries, and
the engine-mode-3 protocol (two self-loading groups per CTA, no producer warp)
is simulated with random timings to check that it always finishes: a group
claims its next task one ahead, issues the task's load at the current tile's
stage-free point unless the task's slab is incomplete, releases its previous S3
tile there, and waits on a slab counter only after releasing everything it
holds. No GPU is used.
"""
import random

import pytest


def decode(slabs, lag, lb, g):
    """s23_decode: claim index -> (kind, slab, index within the slab's tiles)."""
    B = 1 << lb
    if g < lag * B:
        return "S3", g >> lb, g & (B - 1)
    g1 = g - lag * B
    if g1 < 2 * B * (slabs - lag):
        pr, r = g1 >> (lb + 1), g1 & (2 * B - 1)
        first = r < B
        return ("S3", lag + pr, r & (B - 1)) if first else ("S2", pr, r & (B - 1))
    g2 = g1 - 2 * B * (slabs - lag)
    return "S2", slabs - lag + (g2 >> lb), g2 & (B - 1)


def host_order(slabs, lag, lb):
    B = 1 << lb
    out = []
    for h in range(slabs + lag):
        if h < slabs:
            out += [("S3", h, i) for i in range(B)]
        if h >= lag:
            out += [("S2", h - lag, i) for i in range(B)]
    return out


@pytest.mark.parametrize("slabs,lb", [(1, 0), (2, 3), (8, 2), (128, 8), (64, 5)])
def test_closed_form_matches_the_host_order(slabs, lb):
    for lag in range(1, slabs + 1):
        order = host_order(slabs, lag, lb)
        assert [decode(slabs, lag, lb, g) for g in range(len(order))] == order


def simulate_self_served(slabs, lag, lb, ctas, seed, release_before_wait=True):
    """Event simulation of engine mode 3; True when every task finishes and every
    slab counter reaches its target, False on a state with no possible progress."""
    rnd = random.Random(seed)
    B = 1 << lb
    n_tasks = 2 * slabs * B
    claimed = [0]
    done = [0] * slabs  # released S3 completions per slab

    def claim():
        v = claimed[0]
        claimed[0] += 1
        return v

    def ready(t):
        kind, v, _ = decode(slabs, lag, lb, t)
        return kind == "S3" or done[v] == B

    groups = [dict(state="start", cur=None, ahead=None, pending=None, loaded_at=None)
              for _ in range(2 * ctas)]
    clock, finished = 0, 0
    while True:
        clock += 1
        progress = False
        for st in rnd.sample(groups, len(groups)):
            s = st["state"]
            if s == "start":
                st["cur"], st["ahead"] = claim(), claim()
                st["state"] = "wait_slab" if st["cur"] < n_tasks else "exit"
                progress = True
            elif s == "wait_slab":  # blocking wait: the group holds nothing unreleased
                assert st["pending"] is None or not release_before_wait
                if ready(st["cur"]):
                    st["loaded_at"] = clock + rnd.randint(1, 4)
                    st["state"] = "wait_load"
                    progress = True
            elif s == "wait_load":
                if clock >= st["loaded_at"]:
                    st["state"] = "compute"
                progress = True  # time passes
            elif s == "compute":
                # stage-free point: next claim one ahead, load unless its slab is incomplete,
                # release the previous S3 tile
                nxt, st["ahead"] = st["ahead"], (claim() if st["ahead"] < n_tasks else n_tasks)
                if st["pending"] is not None:
                    done[st["pending"]] += 1
                    st["pending"] = None
                kind, v, _ = decode(slabs, lag, lb, st["cur"])
                finished += 1
                if kind == "S3":
                    st["pending"] = v
                if nxt >= n_tasks:
                    st["state"] = "exit"
                elif ready(nxt):
                    st["cur"], st["loaded_at"], st["state"] = nxt, clock + rnd.randint(1, 4), "wait_load"
                else:
                    # deferred: release before waiting on the slab
                    if st["pending"] is not None and release_before_wait:
                        done[st["pending"]] += 1
                        st["pending"] = None
                    st["cur"], st["state"] = nxt, "wait_slab"
                progress = True
            elif s == "exit":
                if st["pending"] is not None:
                    done[st["pending"]] += 1
                    st["pending"] = None
                st["state"] = "gone"
                progress = True
        if all(g["state"] == "gone" for g in groups):
            return finished == n_tasks and all(d == B for d in done)
        if not progress:
            return False


def test_self_served_groups_always_finish():
    rnd = random.Random(7)
    for seed in range(200):
        slabs = rnd.choice([1, 2, 4, 8, 32])
        lag = rnd.randint(1, slabs)
        lb = rnd.choice([0, 1, 2, 4])
        ctas = rnd.choice([1, 2, 5, 37])
        assert simulate_self_served(slabs, lag, lb, ctas, seed), (seed, slabs, lag, lb, ctas)


def test_waiting_while_holding_a_release_can_deadlock():
    """The model detects the hazard the protocol avoids: a group that waits on a
    slab counter while it still owes the release of its own S3 tile of that slab
    stalls forever in some schedule (one CTA, one-slab lag)."""
    outcomes = [simulate_self_served(4, 1, 1, 1, seed, release_before_wait=False) for seed in range(200)]
    assert not all(outcomes)
