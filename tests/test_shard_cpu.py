"""One scan job split across two gloo ranks on CPU (no GPU).

Each rank scans its cost-balanced share of the job's windows -- with the
oracle standing in for the GPU scanner, since this machine has no GPU -- and
rank 0 gathers and finalizes.  The union after finalize must equal a
single-process scan of the whole job, hit for hit and in the same order."""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "tests"))

from infernox_b200 import _native as N  # noqa: E402
from infernox_b200 import shard  # noqa: E402


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _job():
    """A small job: 10 windows of uneven length over one residue buffer."""
    from helpers import frame, models, planted_seq
    cm, g, l = models("small0")
    rng = np.random.default_rng(77)
    lens = [int(x) for x in rng.integers(20, 700, 10)]
    frames, wins, off = [], [], 0
    for k, L in enumerate(lens):
        f = frame(planted_seq(cm, L, 0.5, 1 if L > 150 else 0, seed=300 + k))
        frames.append(f)
        wins.append((off, 1, L))
        off += len(f)
    buf = np.concatenate(frames)
    W = np.array(wins, dtype=N.WINDOW_DTYPE)
    return l, buf, W


def _oracle_batch(cfg, buf):
    """scan_batch stand-in: the oracle, window by window, as BATCH_HIT rows."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    def scan_batch(sub):
        rows = []
        for w, (o, i0, j0) in enumerate(sub.tolist()):
            hits, _, _, _ = oracle.qdb_scan(cfg, 1, 2, buf[o:o + j0 + 2], i0, j0, -5.0, True)
            rows += [(w, h[0], h[1], h[2], h[3]) for h in hits]
        return np.array(rows, dtype=N.BATCH_HIT_DTYPE)

    return scan_batch


def _rank_main(rank, world, port, q):
    import datetime

    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        cfg, buf, W = _job()
        cost = shard.window_cost_fn(cfg, 1, 2)(W["j0"] - W["i0"] + 1)
        parts = shard.split_windows(cost, world)
        mine = shard.scan_shard(_oracle_batch(cfg, buf), W, parts[rank])
        got = shard.gather_hits(dist, mine, rank, world)
        if rank == 0:
            q.put(("job", shard.finalize(got).tobytes(), [p.tolist() for p in parts]))
        q.put(("rank", rank, parts[rank].tolist()))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_two_ranks_union_equals_single_rank():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    msgs = [q.get(timeout=180) for _ in range(3)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    job = [m for m in msgs if m[0] == "job"][0]
    ranks = sorted(m[1:] for m in msgs if m[0] == "rank")
    # each rank scanned exactly the split's share; together every window once
    assert [r[1] for r in ranks] == job[2]
    assert sorted(sum(job[2], [])) == list(range(10))
    cfg, buf, W = _job()
    single = _oracle_batch(cfg, buf)(W)
    got = np.frombuffer(job[1], N.BATCH_HIT_DTYPE)
    assert len(single) > 0
    assert got.tobytes() == single.tobytes()


def test_split_is_balanced_and_deterministic():
    rng = np.random.default_rng(5)
    costs = rng.lognormal(10, 1.0, 500)
    parts = shard.split_windows(costs, 8)
    assert sorted(np.concatenate(parts).tolist()) == list(range(500))
    loads = [costs[p].sum() for p in parts]
    # longest-processing-time-first: no rank exceeds the mean by more than the
    # largest single window
    assert max(loads) - np.mean(loads) <= costs.max()
    assert all(np.array_equal(a, b) for a, b in zip(parts, shard.split_windows(costs, 8)))
    one = shard.split_windows(costs, 1)
    assert len(one) == 1 and one[0].tolist() == list(range(500))


def test_window_cost_matches_count_work():
    from helpers import models
    cm, g, l = models("small2")
    f = shard.window_cost_fn(l, 1, 0)
    for L in (1, 5, l.W - 1, l.W, l.W + 1, 3 * l.W + 7):
        assert f([L])[0] == pytest.approx(l.count_work(1, 0, L)[0], rel=0, abs=0.5)
