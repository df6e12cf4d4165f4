"""One scan job over several GPUs: one process per GPU, windows split across
ranks, hits gathered to rank 0.

Windows -- a sequence's chunk on one strand -- are independent: the
reference schedules them as separate rayon tasks (src/cm_search.rs:1312-1315)
and removes overlaps per window before anything crosses windows
(src/cm_nohmm.rs:759-762).  So a job's window list is split across ranks with
no exchange during the scan:

* ``split_windows``: a static cost-balanced split.  Windows in descending
  order of their exact DP cell count (ties by window index) each go to the
  rank with the least cost so far (ties to the lower rank) -- longest
  processing time first.  Every rank computes the same split from the same
  window list, so no message is needed to agree on it.
* ``scan_shard``: a rank scans its windows in one batched launch and labels
  each hit with its window's index in the job.
* ``gather_hits`` + ``finalize``: the one exchange.  Rank 0 collects every
  rank's hits (torch.distributed gather; NCCL or gloo) and orders them by job
  window index, keeping each window's hits in the scanner's order.  The
  result equals a single-rank scan of the whole job.
"""
from __future__ import annotations

import numpy as np

from . import _native as N


def window_cost_fn(cm, semiring: int, qdbidx: int):
    """Exact DP cells of a window of length L as a vectorised function of L:
    columns up to W from a table (jrow grows), then a constant per column."""
    W = int(cm.W)
    head = np.zeros(W + 1, np.float64)
    for L in range(1, W + 1):
        head[L] = cm.count_work(semiring, qdbidx, L)[0]
    per_col = cm.count_work(semiring, qdbidx, W + 1)[0] - head[W]

    def cost(lengths):
        Ls = np.asarray(lengths, np.int64)
        c = head[np.minimum(Ls, W).clip(0)]
        return c + np.maximum(Ls - W, 0) * per_col

    return cost


def split_windows(costs, world: int) -> list:
    """Per rank, the job indices of its windows (ascending)."""
    costs = np.asarray(costs, np.float64)
    order = sorted(range(len(costs)), key=lambda k: (-costs[k], k))
    load = np.zeros(world, np.float64)
    parts = [[] for _ in range(world)]
    for k in order:
        r = int(np.argmin(load))  # first minimum: ties go to the lower rank
        parts[r].append(k)
        load[r] += costs[k]
    return [np.array(sorted(p), np.int64) for p in parts]


def scan_shard(scan_batch, windows: np.ndarray, idx: np.ndarray) -> np.ndarray:
    """scan_batch(sub_windows) -> BATCH_HIT_DTYPE hits numbered within
    sub_windows; returns them numbered by job window index."""
    sub = np.ascontiguousarray(windows[idx])
    if len(sub) == 0:
        return np.zeros(0, N.BATCH_HIT_DTYPE)
    hits = scan_batch(sub)
    out = hits.copy()
    out["win"] = idx[hits["win"]]
    return out


def gather_hits(dist, hits: np.ndarray, rank: int, world: int):
    """Rank 0 receives every rank's hits (a list indexed by rank); the other
    ranks receive None.  dist is torch.distributed after init_process_group."""
    if dist is None or world == 1:
        return [hits]
    payload = hits.tobytes()
    got = [None] * world if rank == 0 else None
    dist.gather_object(payload, got, dst=0)
    if rank != 0:
        return None
    return [np.frombuffer(b, N.BATCH_HIT_DTYPE).copy() for b in got]


def finalize(parts: list) -> np.ndarray:
    """All ranks' hits in job window order; within a window the scanner's order."""
    if not parts:
        return np.zeros(0, N.BATCH_HIT_DTYPE)
    allh = np.concatenate(parts)
    order = np.argsort(allh["win"], kind="stable")
    return allh[order]
