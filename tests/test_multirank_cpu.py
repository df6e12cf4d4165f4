"""The multi-GPU path of bench.py on CPU: two gloo ranks.

Windows are independent, so ranks share no data; each rank scans its own
seeded batch of the same shape (weak scaling) and the job's figures are the
slowest rank's times and the sum of all ranks' cells.  This runs that
aggregation and the per-rank batch construction in two processes over gloo
on 127.0.0.1 -- no GPU."""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, q):
    import datetime

    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        r, w, lr = bench.env_rank()
        wl = bench.WORKLOADS["batched-uneven-max"]
        buf, wins, lens = bench.make_batch(wl, 8, seed=1000 + r)
        total, e2e, cells = bench.aggregate_ranks(dist, 100.0 + 10 * r, 200.0 - 10 * r, 1e6 * (r + 1), device="cpu")
        q.put((r, w, lr, total, e2e, cells, len(wins), int(lens.sum()), int(buf[:64].sum())))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_two_gloo_ranks_aggregate_and_shard():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, w0, l0, t0, e0, c0, n0, s0, h0), (r1, w1, l1, t1, e1, c1, n1, s1, h1) = out
    assert (r0, r1, w0, w1, l0, l1) == (0, 1, 2, 2, 0, 1)
    # slowest rank's times, all ranks' cells, identical on every rank
    assert t0 == t1 == 110.0 and e0 == e1 == 200.0 and c0 == c1 == 3e6
    # weak scaling: same number of windows per rank, different seeded sequences
    assert n0 == n1 == 16
    assert (s0, h0) != (s1, h1)
