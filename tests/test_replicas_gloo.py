"""Multi-GPU form of the bench (`--gpus N`): independent replicas, one trap per
rank, no collective on the data path; the job's time is the slowest rank's
(max over ranks) and its value the units of all ranks over that time. The
host-side logic runs here as two gloo ranks on the CPU (the GPU form uses the
same functions over NCCL)."""
import os
import socket

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import sys
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "bernasconi-krylov_b200"))
    import datetime
    import torch.distributed as dist
    import bench
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    bits, e0 = bench.replica_trap(16, rank, n_descents=200, quantile=0.05)
    seconds = 1.0 + rank  # the slower rank sets the job's time
    t = bench.max_over_ranks(seconds, world, "cpu")
    out.put((rank, bits, e0, t, bench.whole_job_value(100.0, world, t)))
    dist.barrier()
    dist.destroy_process_group()


def test_replicas_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, b0, e00, t0, v0), (r1, b1, e01, t1, v1) = res
    assert (r0, r1) == (0, 1)
    assert t0 == t1 == 2.0  # max over ranks
    assert v0 == v1 == 100.0 * 2 / 2.0
    # each replica has its own seeded trap, reproducible from its rank alone
    import sys
    sys.path.insert(0, os.path.join(ROOT, "bernasconi-krylov_b200"))
    import bk_b200 as bk
    assert (b0, e00) == bk.select_trap(16, 42, 200, 0.05)
    assert (b1, e01) == bk.select_trap(16, 43, 200, 0.05)
