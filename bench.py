"""Benchmark of the batched QDB/Inside window scan (one JSON line on rank 0).

Other workloads (--workload): "nohmm-cyk-filter" (QDB1 CYK over 100 kb
chunks), "cfg3-cyk" (the 1,500-column, 25-bifurcation model shape: QDB1 CYK
over 1 kb windows, batched against one launch per window), and the
filter/banded stages of the default pipeline --
"f1-ssv" (SSV windows over 100 kb chunks, both strands, of a 4.6 Mb
sequence, F1 = 0.35), "f2-vit" (Viterbi filter over F1-sized windows),
"f3-fwd" (local Forward filter and its composition-bias null over the same
windows), "f3-cascade" (the whole F1 -> F3b pass of f3_filter_sequence over
the 4.6 Mb sequence), "hb-cyk" / "hb-inside" (HMM-banded CYK / float Inside over envelopes with
CP9-shaped bands), "hb-trcyk" (truncated HMM-banded CYK, 5'-and-3' pass, all
four planes), "trq-inside" / "trq-cyk" (the truncated non-banded integer
TrInside / QDB1 TrCYK window scan, 5'-and-3' pass, over short sequences that
hold a homolog cut at both ends) -- each with the oracle timed on the host
cores beside it.

Workload (default "batched-uneven-max"): the batched uneven-window Inside scan
of the --max path.  One 120-consensus-column CM with 3 bifurcations (seeded
synthetic, local configuration), sequences with log-normal lengths clipped to
[200, 20000] nt (median 1.5 kb, i.i.d. 45% GC, a tenth of them carrying one
homolog sampled from the model), both strands, every window
scanned with the non-banded integer Inside scanner (final_stage_inside_opt
with nonbanded=true).  A step is one pass over a batch of --batch sequences
(both strands) drawn from that distribution; each rank scans its own batch
(weak scaling).  The metric is DP cells per second (the reference's cells,
counted exactly from the bands), whole job.

value   device-resident batch: residues already in HBM, hits returned to the host.
e2e     the public API with host buffers: residues copied host->device inside
        the timed region, hit list copied back.
Timing: CUDA events on the stream the library launches on, W warm-up steps,
L2 flushed (256 MB write) before every timed step, max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    # name: (clen, paired fraction, bifurcations, structure seed, param seed,
    #        semiring, band set, median length, sigma, lo, hi, gc)
    # sigma 0.78: about 99% of log-normal lengths with median 1500 fall in [200, 20000]
    "batched-uneven-max": dict(clen=120, paired=0.5, nbif=3, sseed=5, pseed=23, semiring=1, band=0,
                               median=1500, sigma=0.78, lo=200, hi=20000, gc=0.45),
    "nohmm-cyk-filter": dict(clen=72, paired=None, nbif=2, sseed=0, pseed=11, semiring=0, band=1,
                             median=100000, sigma=0.0, lo=100000, hi=100000, gc=0.50),
    # the bifurcation-heavy model shape (1,500 columns, 60% paired, 25
    # bifurcations, W = 1,551): the QDB1 CYK filter scan over 1 kb windows,
    # batched against the plain one-launch-per-window path
    "cfg3-cyk": dict(clen=1500, paired=0.6, nbif=25, sseed=31, pseed=33, semiring=0, band=1,
                     median=1000, sigma=0.0, lo=1000, hi=1000, gc=0.45),
}
FILTER_WORKLOADS = ("f1-ssv", "f2-vit", "f3-fwd", "f3-cascade", "hb-cyk", "hb-inside", "hb-trcyk", "trq-inside", "trq-cyk")
OPS_PER_TERM = {0: 2.0, 1: 7.0}   # CYK: FADD + select; Inside: 6 INT + 1 LDS
OPS_PER_CELL = 2.0                # emission add + store
CUTOFF_BITS = 15.0                # stands in for the E-value threshold
# DRAM bytes (read + write) per DP cell of the scan kernel, from one ncu
# capture of this bench's default step (profiles/qdb_scan_inside_nonbanded_
# traffic.txt: 1.438e12 bytes over 1.058e11 cells in one launch); the
# roofline's traffic is this times the cells of a launch
TRAFFIC_B_PER_CELL = {("level", 1, 0): 13.59}


def env_rank():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)),
            int(os.environ.get("LOCAL_RANK", 0)))


def aggregate_ranks(dist, total_ms, e2e_ms, cells, device="cuda"):
    """Whole-job figures over the ranks (weak scaling, no data exchange): the
    slowest rank's device times (max) and the cells of all ranks (sum).
    dist is torch.distributed after init_process_group, or None for one rank."""
    if dist is None:
        return total_ms, e2e_ms, cells
    import torch
    t = torch.tensor([total_ms, e2e_ms, cells], dtype=torch.float64, device=device)
    tmax = t.clone()
    dist.all_reduce(tmax, op=dist.ReduceOp.MAX)
    tsum = t.clone()
    dist.all_reduce(tsum, op=dist.ReduceOp.SUM)
    return tmax[0].item(), tmax[1].item(), tsum[2].item()


PLANT_FRACTION = 0.1  # sequences that carry one homolog sampled from the model


def make_cm(w):
    from infernox_b200 import synth
    if w["paired"] is None:
        ss = synth.trna_like()
    else:
        ss = synth.structure(w["clen"], w["paired"], w["nbif"], w["sseed"])
    return synth.synth_cm(ss, w["pseed"], name="bench")


def make_model(w):
    from infernox_b200 import model
    return model.configure(make_cm(w), local=True)


def make_batch(w, nseq, seed):
    """Concatenated window frames for nseq sequences, top and bottom strand;
    PLANT_FRACTION of them carry one homolog sampled from the model at a
    random place (lengths, and so cells, are unchanged)."""
    from infernox_b200 import synth
    rng = np.random.default_rng(seed)
    cm = make_cm(w)
    if w["sigma"] > 0:
        lens = np.clip(rng.lognormal(np.log(w["median"]), w["sigma"], nseq), w["lo"], w["hi"]).astype(int)
    else:
        lens = np.full(nseq, w["median"], int)
    frames, wins, off = [], [], 0
    for L in lens:
        top = synth.random_dsq(int(L), w["gc"], rng)
        if rng.random() < PLANT_FRACTION:
            h = synth.emit(cm, rng)
            if 0 < len(h) < L:
                p = int(rng.integers(0, int(L) - len(h) + 1))
                top[p:p + len(h)] = h
        for s in (top, synth.revcomp(top)):
            f = np.concatenate([[255], s, [255]]).astype(np.uint8)
            frames.append(f)
            wins.append((off, 1, int(L)))
            off += len(f)
    buf = np.concatenate(frames)
    W = np.array(wins, dtype=[("dsq_offset", np.int64), ("i0", np.int32), ("j0", np.int32)])
    return buf, W, lens


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": len(self.rows)}
        sm = [float(r[1]) for r in self.rows if len(r) >= 8 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) >= 8 and r[2].replace(".", "").isdigit()]
        if sm:
            out["sm_mhz"] = statistics.median(sm)
            out["sm_max_mhz"] = max(mx) if mx else None
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for k, n in enumerate(names):
            if any(len(r) >= 8 and r[4 + k].lower() == "active" for r in self.rows):
                out["reasons"].append(n)
        return out


def cpu_baseline(cm, w, buf, wins, budget_s):
    """The oracle (C restatement of the reference scanner, built -O3
    -march=native on this host) on all host cores, threads over windows.

    Every thread takes windows of the batch in a seeded random order until
    the time budget is spent; a window started before the deadline is
    finished (the longest, 20 kb, takes a few seconds on one core), and the
    rate is the cells of all finished windows over the elapsed time."""
    oracle = _oracle()
    cores = os.cpu_count() or 1
    perm = [int(k) for k in np.random.default_rng(7).permutation(len(wins))]
    lock = threading.Lock()
    state = {"next": 0, "cells": 0.0, "res": 0, "n": 0, "maxlen": 0}
    deadline = time.perf_counter() + budget_s

    rates = [0.0] * cores

    def worker(t):
        mine, t_start = 0.0, time.perf_counter()
        while time.perf_counter() < deadline:
            with lock:
                if state["next"] >= len(perm):
                    break
                k = perm[state["next"]]
                state["next"] += 1
            o, i0, j0 = wins[k]
            oracle.qdb_scan(cm, w["semiring"], w["band"], buf[o:o + j0 + 2], i0, j0, CUTOFF_BITS, True)
            c, _ = cm.count_work(w["semiring"], w["band"], j0 - i0 + 1)
            mine += c
            with lock:
                state["cells"] += c
                state["res"] += j0 - i0 + 1
                state["n"] += 1
                state["maxlen"] = max(state["maxlen"], j0 - i0 + 1)
        # this thread's own rate: its cells over the time it was busy
        rates[t] = mine / max(time.perf_counter() - t_start, 1e-9)

    t0 = time.perf_counter()
    ths = [threading.Thread(target=worker, args=(t,)) for t in range(cores)]
    for t in ths:
        t.start()
    for t in ths:
        t.join()
    dt = time.perf_counter() - t0
    tot, res, n = state["cells"], state["res"], state["n"]
    # all cores busy: the sum of the threads' own rates (the last windows of
    # a sample finish at different times; counting each thread over its own
    # busy time keeps that tail from diluting the rate)
    return {"value": sum(rates) / 1e9, "unit": "Gcells/s", "cores": cores, "kind": "port",
            "build": "gcc -O3 -march=native -ffp-contract=off",
            "sample": f"{n} windows in seeded random order, every length (longest {state['maxlen']} nt; "
                      f"{res} residues, {tot:.3e} cells) from the same batch, {dt:.1f} s on {cores} threads",
            "windows_per_s": n / dt, "cells": tot, "seconds": dt}


def _renumber(hits, idx):
    """Batch hits numbered within a rank's windows -> numbered by job window."""
    out = hits.copy()
    out["win"] = np.asarray(idx)[hits["win"]]
    return out


def _oracle():
    """The oracle, the -march=native build (the timed CPU baseline)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    if oracle._lib is None:
        oracle.use_native()
    oracle.lib()
    return oracle


def config2_job(sc, cm, w, nseq, check, stream, flush):
    """The batched-uneven-windows workload as stated: `nseq` sequences, both
    strands, every window in ONE persistent launch (device-resident
    residues).  A seeded sample of `check` windows is scanned by the oracle
    and must give the same hits."""
    import torch
    oracle = _oracle()
    buf, wins, lens = make_batch(w, nseq, seed=4242)
    d_buf = torch.from_numpy(buf).cuda()
    sr, band = w["semiring"], w["band"]
    flush.fill_(1)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    hits = sc.scan_batch(sr, band, buf, wins, CUTOFF_BITS, True, device_buf=d_buf.data_ptr())
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    st = sc.stats()
    rng = np.random.default_rng(99)
    sample = sorted(rng.choice(len(wins), size=min(check, len(wins)), replace=False).tolist())
    same = True
    for k in sample:
        o, i0, j0 = (int(x) for x in wins[k])
        ref, _, _, _ = oracle.qdb_scan(cm, sr, band, buf[o:o + j0 + 2], i0, j0, CUTOFF_BITS, True)
        mine = hits[hits["win"] == k]
        got = [(int(h["i"]), int(h["j"]), h["score"].tobytes(), h["bias"].tobytes()) for h in mine]
        exp = [(r[0], r[1], np.float32(r[2]).tobytes(), np.float32(r[3]).tobytes()) for r in ref]
        same = same and got == exp
    if not same:
        raise RuntimeError("full-job hits differ from the oracle on the checked windows")
    del d_buf
    return {"sequences": int(nseq), "windows": int(len(wins)), "residues": int(2 * lens.sum()),
            "launches": int(st["kernel_launches"]), "ms": ms, "kernel_ms": st["kernel_ms"],
            "value": st["cells"] / (ms / 1e3) / 1e9, "unit": "Gcells/s",
            "seq_per_s": nseq / (ms / 1e3), "cells": st["cells"], "hits": int(len(hits)),
            "oracle_checked_windows": len(sample), "oracle_identical": bool(same),
            "timing": "one launch, CUDA events on the library's stream, L2 flushed before"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="batched-uneven-max",
                    choices=sorted(WORKLOADS) + list(FILTER_WORKLOADS) + ["serve", "calibrate"])
    ap.add_argument("--batch", type=int, default=500, help="sequences per step per rank")
    ap.add_argument("--calib-mb", type=float, default=1.6, help="calibrate: Mb of random sequence (-L)")
    ap.add_argument("--models", type=int, default=200, help="serve: CMs in the library")
    ap.add_argument("--requests", type=int, default=12, help="serve: queries")
    ap.add_argument("--rate", type=float, default=200.0, help="serve: Poisson arrivals per second")
    ap.add_argument("--serve-budget", type=int, default=8_000_000, help="serve: active residues (both strands)")
    ap.add_argument("--serve-check", type=int, default=2, help="serve: requests checked alone vs mixed")
    ap.add_argument("--kernel", default="auto", choices=["auto", "level", "sweep"],
                    help="QDB scan kernel (CMGPU_KERNEL_*)")
    ap.add_argument("--job-seqs", type=int, default=10000,
                    help="sequences of the full one-launch job measured once at N=1 (0: skip)")
    ap.add_argument("--job-check", type=int, default=24, help="windows of the full job checked by the oracle")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--plain-windows", type=int, default=16)
    ap.add_argument("--envelopes", type=int, default=2000, help="envelopes per step (HB workloads)")
    args = ap.parse_args()
    if args.workload in FILTER_WORKLOADS:
        return filter_main(args)
    if args.workload == "serve":
        return serve_main(args)
    if args.workload == "calibrate":
        return calibrate_main(args)
    w = WORKLOADS[args.workload]
    rank, world, local_rank = env_rank()
    cm = make_model(w)
    # one job of world x batch sequences; every rank scans its cost-balanced
    # share of the job's windows (infernox_b200.shard) and rank 0 gathers the
    # hits: per-rank work stays fixed as ranks are added (weak scaling)
    from infernox_b200 import shard
    job_buf, job_wins, job_lens = make_batch(w, args.batch * world, seed=1000)
    parts = shard.split_windows(
        shard.window_cost_fn(cm, w["semiring"], w["band"])(job_wins["j0"] - job_wins["i0"] + 1), world)
    mine = parts[rank]
    frames, wl, off = [], [], 0
    for k in mine:
        o, i0, j0 = (int(x) for x in job_wins[k])
        frames.append(job_buf[o:o + j0 + 2])
        wl.append((off, i0, j0))
        off += j0 + 2
    buf = np.concatenate(frames)
    wins = np.array(wl, dtype=job_wins.dtype)
    config = {"workload": args.workload, "model": f"synthetic CM clen={cm.clen} M={cm.M} W={cm.W}",
              "scan": {0: "CYK f32", 1: "Inside i32"}[w["semiring"]] + " " +
                      {0: "non-banded", 1: "QDB1", 2: "QDB2"}[w["band"]],
              "sequences_per_step_per_rank": int(args.batch), "windows_per_step_per_rank": int(len(wins)),
              "residues_per_step_per_rank": int((wins["j0"] - wins["i0"] + 1).sum()),
              "sequences_per_step_job": int(args.batch * world), "cutoff_bits": CUTOFF_BITS,
              "lengths": f"log-normal median {w['median']} sigma {w['sigma']} clipped to [{w['lo']}, {w['hi']}], "
                         f"both strands",
              "homologs": f"{PLANT_FRACTION:.0%} of the sequences carry one homolog sampled from the model",
              "parallelism": f"dp{world}: cost-balanced window split, hits gathered to rank 0",
              "l2": "flushed (256 MB write) before each timed step"}

    if args.impl == "reference":
        if rank != 0:
            return
        per_step = max(2.0, args.cpu_seconds / max(1, args.steps))
        for _ in range(args.warmup):
            cpu_baseline(cm, w, buf, [tuple(x) for x in wins], per_step)
        samples = [cpu_baseline(cm, w, buf, [tuple(x) for x in wins], per_step) for _ in range(args.steps)]
        cells, secs = sum(x["cells"] for x in samples), sum(x["seconds"] for x in samples)
        rate = sum(x["value"] * x["seconds"] for x in samples) / secs
        cb = {"value": rate, "unit": "Gcells/s", "cores": samples[0]["cores"], "kind": "port",
              "build": samples[0]["build"],
              "sample": f"{args.steps} steps of about {per_step:.1f} s, each a seeded random sample of the "
                        f"batch's windows of every length on {samples[0]['cores']} threads (after "
                        f"{args.warmup} warm-up samples); rate = sum of the threads' own rates"}
        line = {"impl": "reference", "metric": "CYK/Inside scan Gcells/s", "value": cb["value"],
                "unit": "Gcells/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": 1e3 * secs / max(1, args.steps),
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
                "data": "synthetic", "config": config, "cpu_baseline": cb,
                "e2e": {"value": cb["value"], "unit": "Gcells/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    import torch
    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    from infernox_b200 import scan
    stream = torch.cuda.current_stream()
    sc = scan.Scanner(cm, device=local_rank, stream=stream.cuda_stream)
    sc.set_kernel({"auto": scan.KERNEL_AUTO, "level": scan.KERNEL_LEVEL, "sweep": scan.KERNEL_SWEEP}[args.kernel])
    d_buf = torch.from_numpy(buf).cuda()
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.int32, device="cuda")
    sr, band = w["semiring"], w["band"]

    def barrier():
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    def step_device():
        return sc.scan_batch(sr, band, buf, wins, CUTOFF_BITS, True, device_buf=d_buf.data_ptr())

    def step_e2e():
        return sc.scan_batch(sr, band, buf, wins, CUTOFF_BITS, True)

    # launch shape tuned on the first 400 windows of the step's batch
    tw = wins[: min(len(wins), 400)]
    tb = buf[: int(tw[-1]["dsq_offset"]) + int(tw[-1]["j0"]) + 2]
    tune = sc.autotune(sr, band, tb, tw, CUTOFF_BITS, device_buf=d_buf.data_ptr())
    for _ in range(args.warmup):
        hits = step_device()
    ref_hits = hits
    clocks = ClockSampler(local_rank)
    barrier()
    clocks.start()
    times, kms, cells, terms, launches, ncand = [], [], 0.0, 0.0, 0, 0
    for _ in range(args.steps):
        flush.fill_(1)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        hits = step_device()
        e1.record(stream)
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
        st = sc.stats()
        kms.append(st["kernel_ms"])
        cells += st["cells"]
        terms += st["terms"]
        launches += st["kernel_launches"]
        ncand += st["candidates"]
    barrier()
    clk = clocks.stop()
    kern_used = sc.stats()["kernel"]
    if not np.array_equal(hits, ref_hits):
        raise RuntimeError("hit lists differ between steps")
    total_ms = sum(times)
    # e2e through the host-buffer API (up to 5 steps)
    e2e_steps = min(args.steps, 5)
    for _ in range(1):
        step_e2e()
    barrier()
    etimes = []
    for _ in range(e2e_steps):
        flush.fill_(1)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        eh = step_e2e()
        e1.record(stream)
        e1.synchronize()
        etimes.append(e0.elapsed_time(e1))
    barrier()
    if not np.array_equal(eh, ref_hits):
        raise RuntimeError("e2e hits differ from the device-resident path")
    e2e_ms = sum(etimes) * args.steps / e2e_steps  # scaled to the timed step count

    total_ms_all, e2e_ms_all, cells_all = aggregate_ranks(dist, total_ms, e2e_ms, cells)

    # the job's hits: every rank's, numbered by job window, gathered to rank 0
    job_hits = shard.finalize(shard.gather_hits(dist, _renumber(ref_hits, mine), rank, world) or [])

    plain = None
    cb = None
    if rank == 0 and args.plain_windows > 0:
        # plain comparator: one launch per window over its own work items, same windows
        k = min(args.plain_windows, len(wins))
        sub = wins[:k]
        sc.scan_batch(sr, band, buf, sub, CUTOFF_BITS, True, plain=True)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ph = sc.scan_batch(sr, band, buf, sub, CUTOFF_BITS, True, plain=True)
        e1.record(stream)
        e1.synchronize()
        pst = sc.stats()
        pms = e0.elapsed_time(e1)
        bh = sc.scan_batch(sr, band, buf, sub, CUTOFF_BITS, True)
        if not np.array_equal(ph, bh):
            raise RuntimeError("plain and batched scans differ")
        plain = {"value": pst["cells"] / (pms / 1e3) / 1e9, "unit": "Gcells/s", "windows": k,
                 "launches": pst["kernel_launches"], "ms": pms}
    job = None
    if rank == 0 and world == 1 and args.job_seqs > 0:
        job = config2_job(sc, cm, w, args.job_seqs, args.job_check, stream, flush)
    if rank == 0:
        if not args.no_cpu:
            cb = cpu_baseline(cm, w, buf, [tuple(x) for x in wins], args.cpu_seconds)

    if rank == 0:
        value = cells_all / (total_ms_all / 1e3) / 1e9
        e2e = cells_all / (e2e_ms_all / 1e3) / 1e9  # e2e_ms is scaled to the same step count
        kernel_ms = sum(kms) / max(1, launches)
        ops_launch = (terms * OPS_PER_TERM[sr] + cells * OPS_PER_CELL) / max(1, launches)
        sm_mhz = clk["sm_mhz"]
        peak_src = "measured SM clock during the timed region"
        if not sm_mhz:
            try:
                sm_mhz = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["sm_max_mhz"]
                peak_src = "MEASURED_PEAKS.json sm_max_mhz"
            except (OSError, KeyError, ValueError):
                sm_mhz, peak_src = 1965.0, "nominal max SM clock"
        nsm = torch.cuda.get_device_properties(local_rank).multi_processor_count
        peak = nsm * 128 * sm_mhz * 1e6 / 1e9  # Gop/s
        achieved = ops_launch / (kernel_ms / 1e3) / 1e9
        kern_name = {1: "level", 2: "sweep"}.get(kern_used, "?")
        step_lat = sorted(times)
        line = {
            "metric": "CYK/Inside scan Gcells/s", "value": value, "unit": "Gcells/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": total_ms_all / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": {0: "f32", 1: "int32"}[sr], "data": "synthetic",
            "config": config,
            "e2e": {"value": e2e, "unit": "Gcells/s",
                    "h2d_bytes_per_step": int(buf.nbytes + len(wins) * 24),
                    # the two device counters, the reportable cells, the hit list
                    "d2h_bytes_per_step": int(8 + ncand / max(1, args.steps) * 16 + len(ref_hits) * 20)},
            "seq_per_s": world * args.batch * args.steps / (total_ms_all / 1e3),
            "step_latency_ms": {"p50": statistics.median(step_lat),
                                "p99": step_lat[min(len(step_lat) - 1, int(0.99 * len(step_lat)))]},
            "gpu_launches": launches,
            "roofline": {"bound": "issue", "achieved": achieved, "peak": peak, "unit": "Gop/s",
                         "frac": achieved / peak,
                         "traffic": (TRAFFIC_B_PER_CELL[(kern_name, sr, band)] * cells / max(1, launches)
                                     if (kern_name, sr, band) in TRAFFIC_B_PER_CELL else None),
                         "traffic_unit": "DRAM bytes per launch (ncu-measured bytes per cell x cells)",
                         "note": f"INT32/FP32 lane-op issue: {nsm} SMs x 128 lanes x {sm_mhz:.0f} MHz "
                                 f"({peak_src}); ops = {OPS_PER_TERM[sr]:.0f}/term + 2/cell"},
            "plain_gpu": plain,
            "batched_over_plain": (value / plain["value"]) if plain else None,
            "cpu_baseline": cb,
            "clocks": clk,
            "launch_shape": {"lanes": tune["best"]["lanes"], "threads": tune["best"]["threads"],
                             "chunk": tune["best"]["chunk"],
                             "tuned_over": [(t["lanes"], t["chunk"], round(t["kernel_ms"], 1))
                                            for t in tune["trials"]]},
            "kernel": kern_name,
            "hits_per_step": int(len(ref_hits)),
            "hits_per_job_step": int(len(job_hits)),
            "e2e_steps": e2e_steps,
            "config2_job": job,
        }
        print(json.dumps(line))
    sc.close()
    if dist:
        dist.destroy_process_group()


# ---------------------------------------------------------------------------
# filter and HMM-banded stages
# ---------------------------------------------------------------------------
# lane-ops per algorithmic cell, for the issue roofline of each kernel:
# SSV: max(dp, xB), +bias (saturating), -cost (floored), row max;
# Viterbi: M 4 adds + 3 max + emission, I 2 adds + max, D 2 adds + max;
# HB: per child relaxation 2 (CYK) or 9 (FLogsum), about 3 children per
# cell, plus emission add and clamp; truncated CYK: the same over the J, L
# and R planes (T only at bifurcations).
FILTER_OPS_PER_CELL = {"f1-ssv": 4.0, "f2-vit": 14.0, "f3-fwd": 16.0, "f3-cascade": 0.0, "hb-cyk": 8.0, "hb-inside": 29.0, "hb-trcyk": 24.0}
FILTER_METRIC = {"f1-ssv": "F1 SSV window scan Gcells/s", "f2-vit": "F2 Viterbi filter Gcells/s",
                 "f3-fwd": "F3 Forward filter Gcells/s (with the F3b bias null)",
                 "f3-cascade": "F1 -> F3b filter pass Mres/s (f3_filter_sequence, both strands)",
                 "hb-cyk": "HMM-banded CYK Gcells/s", "hb-inside": "HMM-banded Inside Gcells/s",
                 "hb-trcyk": "truncated HMM-banded CYK Gcells/s (band cells, 4 planes each)",
                 "trq-inside": "truncated non-banded TrInside Gcells/s (J-plane cells, 4 planes each)",
                 "trq-cyk": "truncated QDB TrCYK Gcells/s (J-plane cells, 4 planes each)"}
FILTER_DTYPE = {"f1-ssv": "u8 (packed s16x2)", "f2-vit": "i16", "f3-fwd": "f32", "f3-cascade": "u8/f32", "hb-cyk": "f32", "hb-inside": "f32",
                "hb-trcyk": "f32", "trq-inside": "i32", "trq-cyk": "f32"}


def trq_work(cfg, qdb, L, fill_t=True):
    """(J-plane cells, child relaxations) of the truncated QDB scan of one
    window of L residues, counted from generic_tr_scan's loops: cnum per cell
    for each non-bifurcation state and the k-splits of B states, on the J, L
    and R planes (and the T plane's splits of B states)."""
    M, W = cfg.M, cfg.W
    w = min(W, L)
    dmax = {0: np.full(M, W), 1: np.asarray(cfg.dmax1), 2: np.asarray(cfg.dmax2)}[qdb]
    dxcap = np.minimum(dmax, W)
    st, stid = np.asarray(cfg.sttype), np.asarray(cfg.stid)
    cnum, cfirst = np.asarray(cfg.cnum), np.asarray(cfg.cfirst)
    live = np.array([v > 0 and st[v] != 7 and not (st[v] in (2, 3, 4, 5) and v + 1 < M and stid[v + 1] == 19)
                     for v in range(M)])
    lv = np.nonzero(live)[0]
    nb, bb = lv[st[lv] != 8], lv[st[lv] == 8]
    cells = terms = 0.0
    for jrow in range(1, w + 1):
        ncol = 1 if jrow < w else L - w + 1
        c = np.minimum(jrow, dxcap[nb])
        cells += ncol * float(c.sum())
        terms += ncol * 3.0 * float((c * cnum[nb]).sum())
        for v in bb:
            cb = min(jrow, int(dxcap[v]))
            y, wl = int(cnum[v]), int(cfirst[v])
            d = np.arange(1, cb + 1)
            k = d + 1 if qdb == 0 else np.maximum(np.minimum(dxcap[y], d) - np.maximum(d - dxcap[wl], 0) + 1, 0)
            cells += ncol * cb
            terms += ncol * float(k.sum()) * (4 if fill_t else 3)
    return cells, terms


def _chunks(total, chunk, rng, cons, nplant, gc):
    """Both strands of a total-residue sequence with planted consensus runs,
    cut into chunk frames."""
    from infernox_b200 import p7, synth
    frames, wins, off = [], [], 0
    top = p7.planted_residues(total, cons, nplant, int(rng.integers(1 << 30)), gc=gc)
    for s in (top, synth.revcomp(top)):
        for a in range(0, total, chunk):
            piece = s[a:a + chunk]
            f = np.concatenate([[255], piece, [255]]).astype(np.uint8)
            frames.append(f)
            wins.append((off, 1, len(piece)))
            off += len(f)
    W = np.array(wins, dtype=[("dsq_offset", np.int64), ("i0", np.int32), ("j0", np.int32)])
    return np.concatenate(frames), W


def _same(out, ref):
    if isinstance(out, np.ndarray):
        return np.array_equal(out.view(np.uint8), ref.view(np.uint8))
    if isinstance(out, tuple):  # bits: overflowed windows score NaN
        return all(np.array_equal(np.ascontiguousarray(a).view(np.uint8), np.ascontiguousarray(b).view(np.uint8))
                   for a, b in zip(out, ref))
    return out == ref


def filter_main(args):
    """One JSON line for the F1 / F2 / HB workloads (rank 0 prints)."""
    from concurrent.futures import ThreadPoolExecutor
    rank, world, local_rank = env_rank()
    kind = args.workload
    rng = np.random.default_rng(4242 + rank)
    from infernox_b200 import hb, model, p7, synth
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    config = {"workload": kind, "parallelism": f"dp{world}", "l2": "flushed (256 MB write) before each timed step"}
    unit, div = ("Mres/s", 1e6) if kind == "f3-cascade" else ("Gcells/s", 1e9)
    if kind in ("f1-ssv", "f2-vit", "f3-fwd", "f3-cascade"):
        M = 120
        prof, cons = p7.synthetic_profile(M, 77, 0.6)
        maxl = int(1.25 * M)
        mmu, mlam, f1 = -8.0, 0.693, 0.35
        if kind == "f3-cascade":
            buf, wins = _chunks(4_600_000, 100_000, rng, cons, 40, 0.508)
            f3, f3b, ftau, flam, cmw = 0.02, 0.02, -6.0, 0.69, 148
            compo = p7.mean_composition(prof)
            config.update({"model": f"synthetic p7 profile M={M} (peak 0.6)",
                           "sequence": "4.6 Mb, both strands, 100 kb chunks, 40 planted consensus runs",
                           "stages": "F1 SSV windows (F1 = 0.35), F3 Forward and F3b bias (0.02, the <2 Mb "
                                     "thresholds), merge", "lftau": ftau, "lflambda": flam, "cmw": cmw})
        elif kind == "f1-ssv":
            buf, wins = _chunks(4_600_000, 100_000, rng, cons, 40, 0.508)
            config.update({"model": f"synthetic p7 profile M={M} (peak 0.6)",
                           "sequence": "4.6 Mb, both strands, 100 kb chunks, 40 planted consensus runs",
                           "f1": f1, "lmmu": mmu, "lmlambda": mlam, "max_length": maxl})
        else:
            buf, wins = _chunks(2_000_000, 2 * maxl, rng, cons, 40, 0.508)
            config.update({"model": f"synthetic p7 profile M={M} (peak 0.6)",
                           "windows": f"{len(wins)} windows of {2 * maxl} residues (2 Mb, both strands)"})
        cells_step = int((wins["j0"] - wins["i0"] + 1).sum()) * (1 if kind == "f3-cascade" else M)
    elif kind in ("trq-inside", "trq-cyk"):
        cmw = WORKLOADS["batched-uneven-max"]
        cm_s = synth.synth_cm(synth.structure(cmw["clen"], cmw["paired"], cmw["nbif"], cmw["sseed"]), cmw["pseed"],
                              name="bench")
        cfg = model.configure(cm_s, local=True)
        frames, wl, off = [], [], 0
        for q in range(args.envelopes):
            h = synth.emit(cm_s, rng)
            c5, c3 = len(h) // 4, len(h) // 5
            seq = np.concatenate([synth.random_dsq(20, 0.45, rng), h[c5:len(h) - c3],
                                  synth.random_dsq(20, 0.45, rng)]).astype(np.uint8)
            f = np.concatenate([[255], seq, [255]]).astype(np.uint8)
            frames.append(f)
            wl.append((off, 1, len(seq)))
            off += len(f)
        buf = np.concatenate(frames)
        wins = np.array(wl, dtype=[("dsq_offset", np.int64), ("i0", np.int32), ("j0", np.int32)])
        trq_qdb = 0 if kind == "trq-inside" else 1
        lens = wins["j0"] - wins["i0"] + 1
        config.update({"model": f"synthetic CM clen={cfg.clen} M={cfg.M} W={cfg.W} (local)",
                       "windows": f"{len(wins)} whole sequences, each a sampled homolog cut by 1/4 at the 5' end "
                                  f"and 1/5 at the 3' end between 20-nt random flanks (median "
                                  f"{int(np.median(lens))} nt)",
                       "pass": "5'-and-3' (PLI_PASS_5P_AND_3P_FORCE), J/L/R/T planes",
                       "bands": "non-banded" if trq_qdb == 0 else "QDB1 (beta1)"})
    else:
        cmw = WORKLOADS["batched-uneven-max"]
        cm_s = synth.synth_cm(synth.structure(cmw["clen"], cmw["paired"], cmw["nbif"], cmw["sseed"]), cmw["pseed"],
                              name="bench")
        cfg = model.configure(cm_s, local=True)
        frames, tasks, off = [], [], 0
        nenv = args.envelopes
        for q in range(nenv):
            h = synth.emit(cm_s, rng)
            n = cfg.W + 40
            seq = synth.random_dsq(n, 0.45, rng)
            p = int(rng.integers(10, max(11, n - len(h) - 10)))
            seq[p - 1:p - 1 + len(h)] = h[: n - p + 1]
            f = np.concatenate([[255], seq, [255]]).astype(np.uint8)
            i0, j0 = 5, 5 + cfg.W - 1
            im, ix, jm, jx = synth.hb_band_rects(cm_s.st, p, i0, j0, 20, rng)
            tasks.append((off, i0, j0, 0.0, 0.0, hb.ij2d_bands(cfg.sttype, im, ix, jm, jx)))
            frames.append(f)
            off += len(f)
        buf = np.concatenate(frames)
        cells_step = sum(int(np.maximum(t[5].hdmax - t[5].hdmin + 1, 0).sum()) for t in tasks)
        config.update({"model": f"synthetic CM clen={cfg.clen} M={cfg.M} W={cfg.W} (local)",
                       "envelopes": f"{nenv} envelopes of W residues, one sampled homolog each, CP9-shaped bands "
                                    "(per-state i/j rectangles of +-20 around the homolog's consensus coordinates)",
                       "band_cells_per_step": cells_step})
    if kind in ("trq-inside", "trq-cyk", "hb-trcyk"):
        tri = hb.tr_inputs(cm_s, cfg, 4, True)
    if kind == "hb-trcyk":
        ones = np.ones(cfg.M, np.uint8)
        valid = (ones, ones, ones, ones)
        config.update({"pass": "5'-and-3' (PLI_PASS_5P_AND_3P_FORCE), J/L/R/T planes", "planes": 4})
    if kind in ("trq-inside", "trq-cyk"):
        per = {}
        for L in lens:
            if int(L) not in per:
                per[int(L)] = trq_work(cfg, trq_qdb, int(L))
        cells_step = int(sum(per[int(L)][0] for L in lens))
        tpc = sum(per[int(L)][1] for L in lens) / max(float(cells_step), 1.0)
        FILTER_OPS_PER_CELL[kind] = tpc * (7.0 if kind == "trq-inside" else 2.0) + 2.0
        config.update({"cells_per_step": cells_step, "child_terms_per_cell": round(tpc, 2)})

    # the oracle on the host cores, one unit (window / envelope) at a time
    import oracle
    oracle.lib()
    if kind == "f1-ssv":
        units = [(int(o), int(j)) for o, _, j in wins]
        one = lambda u: oracle.f1_msv_windows(M, prof.mat, prof.trans, maxl, mmu, mlam, buf, [u[0]], [u[1]], f1,
                                              maxl) and u[1] * M
    elif kind == "f2-vit":
        # 64 windows per oracle call: the filter is built once per call, as the
        # reference builds it once per search
        units = [(wins["dsq_offset"][a:a + 64].astype(np.int64), wins["j0"][a:a + 64].astype(np.int32))
                 for a in range(0, len(wins), 64)]
        one = lambda u: oracle.vit_score_batch(M, prof.mat, prof.trans, buf, u[0], u[1]) and int(u[1].sum()) * M
    elif kind == "f3-cascade":
        units = [(int(o), int(j)) for o, _, j in wins]

        def one(u):
            oracle.f3_filter_sequence((M, prof.mat, prof.trans), compo, ftau, flam, buf[u[0]:u[0] + u[1] + 2], f1,
                                      f3, f3b, cmw, max_length=maxl, mmu=mmu, mlambda=mlam)
            return u[1]
    elif kind == "f3-fwd":
        # 64 windows per oracle call (the SSE2 engine, the reference's x86 path)
        units = [(wins["dsq_offset"][a:a + 64].astype(np.int64), wins["j0"][a:a + 64].astype(np.int32))
                 for a in range(0, len(wins), 64)]
        compo = p7.mean_composition(prof)

        def one(u):
            oracle.fwd_score_batch(M, prof.mat, prof.trans, buf, u[0], u[1])
            oracle.bias_score_batch(compo, M, buf, u[0], u[1])
            return int(u[1].sum()) * M
    elif kind in ("trq-inside", "trq-cyk"):
        units = list(range(len(wins)))
        ttab = {"lmesc": tri.lmesc, "rmesc": tri.rmesc, "pty": tri.pty, "ilmesc": tri.ilmesc, "irmesc": tri.irmesc,
                "ipty": tri.ipty, "lpos": tri.lpos, "rpos": tri.rpos, "clen": tri.clen}

        def one(q):
            o, i0, j0 = (int(x) for x in wins[q])
            oracle.trq_scan(cfg, kind == "trq-inside", ttab, buf[o:o + j0 + 2], i0, j0, 0.0, True, trq_qdb, 4, True)
            return int(per[j0 - i0 + 1][0])
    elif kind == "hb-trcyk":
        units = list(range(len(tasks)))
        ttab = {"lmesc": tri.lmesc, "rmesc": tri.rmesc, "pty": tri.pty, "lpos": tri.lpos, "rpos": tri.rpos,
                "clen": tri.clen}

        def one(q):
            o, i0, j0, ec, cut, b = tasks[q]
            oracle.tr_hb_scan(cfg, False, ttab, valid, (b.jmin, b.jmax, b.hd_off, b.hdmin, b.hdmax),
                              buf[o:o + j0 + 2], i0, j0, cut, True, 4, ec, True)
            return int(np.maximum(b.hdmax - b.hdmin + 1, 0).sum())
    else:
        units = list(range(len(tasks)))

        def one(q):
            o, i0, j0, ec, cut, b = tasks[q]
            oracle.hb_scan(cfg, kind == "hb-inside", (b.jmin, b.jmax, b.hd_off, b.hdmin, b.hdmax),
                           buf[o:o + j0 + 2], i0, j0, ec, True, cut, True)
            return int(np.maximum(b.hdmax - b.hdmin + 1, 0).sum())
    cores = os.cpu_count() or 1
    perm = np.random.default_rng(7).permutation(len(units))
    pos = {"at": 0}

    def cpu_sample(budget_s):
        """Units of one step's inputs (seeded random order, continuing where
        the last sample stopped) on every host core until budget_s passes."""
        lock = threading.Lock()
        st = {"n": 0, "cells": 0}
        deadline = time.perf_counter() + budget_s

        def worker():
            while time.perf_counter() < deadline:
                with lock:
                    u = units[int(perm[pos["at"] % len(units)])]
                    pos["at"] += 1
                    st["n"] += 1
                c = one(u)
                with lock:
                    st["cells"] += c
        t0 = time.perf_counter()
        with ThreadPoolExecutor(cores) as ex:
            for _ in range(cores):
                ex.submit(worker)
        dt = time.perf_counter() - t0
        return {"value": st["cells"] / dt / div, "unit": unit, "cores": cores, "kind": "port",
                "sample": f"{st['n']} of {len(units)} units of one step's inputs, {dt:.1f} s on {cores} threads",
                "cells": st["cells"], "seconds": dt}

    if args.impl == "reference":
        if rank != 0:
            return
        per_step = max(1.0, args.cpu_seconds / max(1, args.steps))
        for _ in range(args.warmup):
            cpu_sample(per_step)
        samples = [cpu_sample(per_step) for _ in range(args.steps)]
        cells, secs = sum(x["cells"] for x in samples), sum(x["seconds"] for x in samples)
        val = cells / secs / div
        cb = {"value": val, "unit": unit, "cores": cores, "kind": "port",
              "sample": f"{args.steps} steps of {per_step:.1f} s, each a bounded sample of one step's units "
                        f"on {cores} threads (after {args.warmup} warm-up samples)"}
        print(json.dumps({"impl": "reference", "metric": FILTER_METRIC[kind], "value": val, "unit": unit,
                          "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                          "ms_per_step": 1e3 * secs / max(1, args.steps), "higher_is_better": True,
                          "scaling": "weak", "vs_baseline": None, "dtype": FILTER_DTYPE[kind], "data": "synthetic",
                          "config": config, "cpu_baseline": cb,
                          "e2e": {"value": val, "unit": unit, "h2d_bytes_per_step": 0,
                                  "d2h_bytes_per_step": 0}}))
        return

    import torch
    torch.cuda.set_device(local_rank)
    stream = torch.cuda.current_stream()
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.int32, device="cuda")
    pinned = torch.from_numpy(buf).pin_memory()  # e2e copies come from pinned host memory
    buf = pinned.numpy()
    if kind == "f1-ssv":
        f = p7.MsvFilter(prof, maxl, mmu, mlam, device=local_rank)
        call = lambda: f.f1_windows_batch(buf, wins, f1, maxl)
        stats = f.stats
        h2d = buf.nbytes + len(wins) * 16
    elif kind == "f2-vit":
        f = p7.VitFilter(prof, device=local_rank)
        call = lambda: f.score_batch(buf, wins)
        stats = lambda: p7.vit_stats(f)
        h2d = buf.nbytes + len(wins) * 24
    elif kind == "f3-cascade":
        mf = p7.MsvFilter(prof, maxl, mmu, mlam, device=local_rank)
        f = p7.FwdFilter(prof, compo, ftau, flam, device=local_rank)
        call = lambda: p7.f3_filter_batch(f, buf, wins, f1, f3, f3b, cmw, mf=mf)[0]
        stats = f.stats
        h2d = 2 * buf.nbytes + len(wins) * 16
    elif kind == "f3-fwd":
        f = p7.FwdFilter(prof, p7.mean_composition(prof), -6.0, 0.69, device=local_rank)
        call = lambda: f.score_batch(buf, wins)
        stats = f.stats
        h2d = buf.nbytes + 2 * len(wins) * 16
    elif kind in ("trq-inside", "trq-cyk"):
        from infernox_b200 import _native as N
        from infernox_b200.scan import Scanner
        sc = Scanner(cfg, device=local_rank)
        sr = N.INSIDE_I32 if kind == "trq-inside" else N.CYK_F32
        call = lambda: hb.tr_qdb_scan_batch(sc, sr, trq_qdb, tri, 4, True, buf, wins, 0.0)
        stats = lambda: hb.tr_qdb_stats(sc)
        call()
        if stats()[1] != cells_step:
            raise RuntimeError("J-plane cell counts of the library and of trq_work differ")
        h2d = buf.nbytes + len(wins) * 16 + cfg.M * (2 * 18 + 1) * 4
    elif kind == "hb-trcyk":
        from infernox_b200.scan import Scanner
        sc = Scanner(cfg, device=local_rank)
        ttasks = [t + (valid,) for t in tasks]
        call = lambda: hb.tr_scan_hb_batch(sc, 0, tri, 4, True, buf, ttasks)
        stats = lambda: hb.hb_stats(sc)
        h2d = buf.nbytes + sum(t[5].hdmin.nbytes + t[5].hdmax.nbytes + 3 * t[5].jmin.nbytes + 4 * cfg.M
                               for t in tasks)
    else:
        from infernox_b200.scan import Scanner
        sc = Scanner(cfg, device=local_rank)
        sr = 0 if kind == "hb-cyk" else 2
        call = lambda: hb.hb_scan_batch(sc, sr, True, True, buf, tasks)
        stats = lambda: hb.hb_stats(sc)
        h2d = buf.nbytes + sum(t[5].hdmin.nbytes + t[5].hdmax.nbytes + 3 * t[5].jmin.nbytes for t in tasks)
    for _ in range(args.warmup):
        ref = call()
    clocks = ClockSampler(local_rank)
    torch.cuda.synchronize()
    clocks.start()
    times, kms, launches = [], [], 0
    for _ in range(args.steps):
        flush.fill_(1)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        out = call()
        e1.record(stream)
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
        ms, _, nl = stats()
        kms.append(ms)
        launches += nl
    torch.cuda.synchronize()
    clk = clocks.stop()
    if not _same(out, ref):
        raise RuntimeError("results differ between steps")
    kernel_ms = sum(kms) / len(kms)
    value = cells_step / (kernel_ms / 1e3) / div
    e2e = cells_step / (statistics.mean(times) / 1e3) / div
    sm_mhz = clk["sm_mhz"] or 1965.0
    nsm = torch.cuda.get_device_properties(local_rank).multi_processor_count
    peak = nsm * 128 * sm_mhz * 1e6 / 1e9
    achieved = FILTER_OPS_PER_CELL[kind] * cells_step / (kernel_ms / 1e3) / 1e9
    cb = cpu_sample(args.cpu_seconds)
    metric = FILTER_METRIC[kind]
    line = {"metric": metric, "value": value, "unit": unit, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": statistics.mean(times), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": FILTER_DTYPE[kind],
            "data": "synthetic", "config": config,
            "e2e": {"value": e2e, "unit": unit, "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": None},
            "gpu_launches": launches,
            "roofline": {"bound": "issue", "achieved": achieved, "peak": peak, "unit": "Gop/s",
                         "frac": achieved / peak, "traffic": None,
                         "note": f"{FILTER_OPS_PER_CELL[kind]:.0f} lane-ops per cell; {nsm} SMs x 128 lanes x "
                                 f"{sm_mhz:.0f} MHz"},
            "cpu_baseline": cb, "clocks": clk}
    if kind == "f3-cascade":
        # several kernels (SSV scan and replay, Forward, bias): the kernel roofline
        # lines belong to f1-ssv and f3-fwd
        line["roofline"] = None
    if rank == 0:
        print(json.dumps(line))


# ---------------------------------------------------------------------------
# serving loop (cmscan-style)
# ---------------------------------------------------------------------------
def serve_library(nmodels, seed=77):
    """nmodels synthetic CMs of 40-400 consensus columns, 30-50% paired,
    0-6 bifurcations (no more than one per 40 columns), local configuration."""
    from infernox_b200 import model, synth
    rng = np.random.default_rng(seed)
    cms, cfgs = [], []
    for k in range(nmodels):
        clen = int(rng.integers(40, 401))
        nb = int(rng.integers(0, min(6, clen // 40) + 1))
        ss = synth.structure(clen, float(rng.uniform(0.3, 0.5)), nb, int(rng.integers(1 << 30)))
        cm = synth.synth_cm(ss, int(rng.integers(1 << 30)), name=f"lib{k}")
        cms.append(cm)
        cfgs.append(model.configure(cm, local=True))
    return cms, cfgs


def serve_requests(cms, n, rate, seed=78):
    """n queries with Poisson arrivals at `rate` per second, lengths
    log-uniform in [100, 100000], GC uniform in [0.4, 0.6], 30% with one
    homolog sampled from a random library model planted at a random place."""
    from infernox_b200 import serve, synth
    rng = np.random.default_rng(seed)
    t, reqs = 0.0, []
    for k in range(n):
        t += float(rng.exponential(1.0 / rate))
        L = int(np.exp(rng.uniform(np.log(100), np.log(100000))))
        seq = synth.random_dsq(L, float(rng.uniform(0.4, 0.6)), rng)
        if rng.random() < 0.3:
            h = synth.emit(cms[int(rng.integers(len(cms)))], rng)
            if 0 < len(h) < L:
                p = int(rng.integers(0, L - len(h)))
                seq[p:p + len(h)] = h
        reqs.append(serve.Request(k, seq, arrival=t))
    return reqs


def serve_main(args):
    rank, world, local_rank = env_rank()
    if rank != 0:
        return
    from infernox_b200 import serve
    t_build = time.perf_counter()
    cms, cfgs = serve_library(args.models)
    t_build = time.perf_counter() - t_build
    reqs = serve_requests(cms, args.requests, args.rate)
    config = {"workload": "serve", "library": f"{len(cfgs)} synthetic CMs, clen 40-400, 0-6 bifurcations, local",
              "requests": len(reqs), "arrivals": f"Poisson, {args.rate:g} per second",
              "query_lengths": "log-uniform 100-100000 nt, both strands; 30% carry one planted homolog",
              "scan": "--nohmm per window: QDB1 CYK filter, QDB2 Inside on its envelopes",
              "cutoffs_bits": {"f6": 12.0, "final": CUTOFF_BITS, "note": "bit cutoffs stand in for the "
                               "E-value thresholds (no calibration)"},
              "residues": int(sum(r.residues for r in reqs)), "library_build_s": round(t_build, 1)}
    if args.impl == "reference":
        # the oracle on the host cores: the per-query, per-model loop of cmscan
        # on a bounded sample (the first requests, all models), one thread per model
        oracle = _oracle()
        from concurrent.futures import ThreadPoolExecutor
        from infernox_b200.synth import revcomp
        cores = os.cpu_count() or 1
        sample = sorted(reqs, key=lambda r: len(r.seq))[: max(1, min(args.steps, 4))]

        def one(k_req):
            k, r = k_req
            for s in (r.seq, revcomp(r.seq)):
                dsq = np.concatenate([[255], s, [255]]).astype(np.uint8)
                envs = oracle.cyk_seq_filter(cfgs[k], dsq, len(s), 12.0, True)
                if envs:
                    oracle.final_stage_inside_opt(cfgs[k], dsq, envs, CUTOFF_BITS, True, False)

        t0 = time.perf_counter()
        with ThreadPoolExecutor(cores) as ex:
            list(ex.map(one, [(k, r) for r in sample for k in range(len(cfgs))]))
        dt = time.perf_counter() - t0
        value = len(sample) / dt
        line = {"impl": "reference", "metric": "served sequences/s (cmscan --nohmm, CM library)", "value": value,
                "unit": "seq/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": 1e3 * dt / max(1, len(sample)), "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32+int32", "data": "synthetic", "config": config,
                "cpu_baseline": {"value": value, "unit": "seq/s", "cores": cores, "kind": "port",
                                 "sample": f"the {len(sample)} shortest queries ({sum(len(r.seq) for r in sample)} nt) "
                                           f"against all {len(cfgs)} models, threads over models"},
                "e2e": {"value": value, "unit": "seq/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    import torch
    torch.cuda.set_device(local_rank)
    srv = serve.Server(cfgs, device=local_rank, budget_residues=args.serve_budget)
    # warm-up: every model's plans built and uploaded by a few short queries
    warm = serve_requests(cms, max(1, args.warmup), 1e6, seed=79)
    t_warm = time.perf_counter()
    for r in warm:
        r.seq = r.seq[:300]
        srv.submit(r)
    while not srv.idle():
        srv.step()
    srv.finished.clear()
    print(f"serve: library of {len(cfgs)} built in {t_build:.1f} s, warm-up pass {time.perf_counter() - t_warm:.1f} s "
          f"(kernel {srv.kernel_ms / 1e3:.1f} s)", file=sys.stderr, flush=True)
    srv.kernel_ms = 0.0
    cells = [0.0]

    def step_counted():
        srv.step()
        for sc in srv.scanners[srv.cursor - 1: srv.cursor] if srv.cursor else srv.scanners[-1:]:
            cells[0] += sc.stats()["cells"]

    # real time: requests enter the queue at their arrival times
    torch.cuda.synchronize()
    srv.t0 = time.perf_counter()
    pending = sorted(reqs, key=lambda r: r.arrival)
    nxt = 0
    steps = 0
    while nxt < len(pending) or not srv.idle():
        now = srv.clock()
        while nxt < len(pending) and pending[nxt].arrival <= now:
            srv.submit(pending[nxt])
            nxt += 1
        if srv.idle():
            time.sleep(max(0.0, min(0.01, pending[nxt].arrival - now)))
            continue
        srv.step()
        steps += 1
        if steps % 50 == 0:
            print(f"serve: {srv.clock():.1f} s, {steps} model steps, {len(srv.active)} active, "
                  f"{len(srv.queue)} queued, {len(srv.finished)} done, kernel {srv.kernel_ms / 1e3:.1f} s",
                  file=sys.stderr, flush=True)
    torch.cuda.synchronize()
    wall = srv.clock()
    done = [r for r in srv.finished if r.status == serve.OK]
    lat = sorted(r.done - r.arrival for r in done)
    span = max(r.done for r in done) - min(r.arrival for r in done)
    value = len(done) / span
    # identity check on a few requests: alone == in the mix
    # (the shortest requests: a request scanned alone takes a full library pass)
    by_len = sorted(done, key=lambda r: len(r.seq))
    same = all(serve.scan_alone(srv, r) == r.hits for r in by_len[: args.serve_check])
    if not same:
        raise RuntimeError("a served request's hits differ from the same request scanned alone")
    # plain comparator: the same queries, one launch per window per stage
    # (scan_alone), timed on a subset
    sub = by_len[: max(1, args.serve_check)]
    t0 = time.perf_counter()
    for r in sub:
        serve.scan_alone(srv, r)
    torch.cuda.synchronize()
    plain_dt = time.perf_counter() - t0
    plain = {"value": len(sub) / plain_dt, "unit": "seq/s", "requests": len(sub),
             "residues": int(sum(r.residues for r in sub)), "s": plain_dt}
    line = {"metric": "served sequences/s (cmscan --nohmm, CM library)", "value": value, "unit": "seq/s",
            "n_gpus": 1, "steps": steps, "warmup": args.warmup, "ms_per_step": 1e3 * wall / max(1, steps),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32+int32",
            "data": "synthetic", "config": config,
            "e2e": {"value": value, "unit": "seq/s", "h2d_bytes_per_step": int(config["residues"] / max(1, steps)),
                    "d2h_bytes_per_step": 0},
            "latency_s": {"p50": statistics.median(lat), "p99": lat[min(len(lat) - 1, int(0.99 * len(lat)))],
                          "max": lat[-1]},
            "residues_per_s": config["residues"] / span,
            "gpu_launches": srv.launches, "model_steps": srv.model_steps, "kernel_s": srv.kernel_ms / 1e3,
            "plain_gpu": plain, "served_over_plain_residue_rate":
                (config["residues"] / span) / (plain["residues"] / plain_dt),
            "identity_checked_requests": min(len(done), args.serve_check)}
    print(json.dumps(line))
    srv.close()



# ---------------------------------------------------------------------------
# cmcalibrate
# ---------------------------------------------------------------------------
def calibrate_main(args):
    """One JSON line for --workload calibrate: cmcalibrate's default run
    (calibrate_cm, src/cm_calibrate.rs:1102) of the 72-column tRNA-like CM --
    L = 1.6 Mb = 160 random genomic 10 kb sequences, QDB bands at beta 1e-15,
    four exp modes (glocal / local x CYK / Inside), null3, tail fits.  A step
    is one whole calibration through cmgpu_calibrate (host generator,
    configuration, four batched scans, fits); each rank calibrates its own
    copy of the model with its own seed (weak scaling, no exchange).

    value  DP cells of the four scans / their device time (library events)
    e2e    the same cells / the wall time of the whole synchronous call"""
    from concurrent.futures import ThreadPoolExecutor
    rank, world, local_rank = env_rank()
    from infernox_b200 import calibrate as cal
    from infernox_b200 import model, synth
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    cm_s = synth.synth_cm(synth.trna_like(), 11, name="cfg0")
    W = model.configure(cm_s, local=False).W
    ccfg = cal.CalibrateConfig(seed=181 + rank, l_mb=args.calib_mb)
    nseq = cal.n_sequences(ccfg)
    g, l = cal.calibration_configs(cm_s, W, ccfg)
    config = {"workload": "calibrate", "model": f"synthetic CM clen={g.clen} M={g.M} W={W} (tRNA-like, "
                                                f"4-stem multibranch)",
              "calibration": f"-L {ccfg.l_mb} Mb = {nseq} random genomic sequences of 10 kb (five-state genomic "
                             f"HMM, seed {ccfg.seed}), QDB2 bands at beta {ccfg.beta:g}, 4 exp modes "
                             f"(glocal/local x CYK/Inside), cutoff -inf, null3, tails gtailn {ccfg.gtailn} / "
                             f"ltailn {ccfg.ltailn}",
              "parallelism": f"dp{world}", "l2": "flushed (256 MB write) before each timed step"}
    # CPU: the oracle's restatement of collect_scores's scan, one (sequence,
    # mode) unit at a time on every host core (the reference runs them on one)
    import oracle
    oracle.lib()
    frames = cal.sample_genomic_sequences(ccfg.seed, cal.EXPTAIL_CHUNKLEN, nseq)
    flen = cal.EXPTAIL_CHUNKLEN + 2
    units = [(s, m) for s in range(nseq) for m in range(4)]
    perm = np.random.default_rng(7).permutation(len(units))
    cores = os.cpu_count() or 1
    pos = {"at": 0}

    def one(u):
        s, m = u
        c = l if cal.exp_mode_is_local(m) else g
        _, cells = oracle.calib_scan(c, int(cal.exp_mode_is_inside(m)), 2, frames[s * flen:(s + 1) * flen], 1,
                                     cal.EXPTAIL_CHUNKLEN, True, want_cells=True)
        return cells

    def cpu_sample(budget_s):
        lock = threading.Lock()
        st = {"n": 0, "cells": 0.0}
        deadline = time.perf_counter() + budget_s

        def worker():
            while time.perf_counter() < deadline:
                with lock:
                    u = units[int(perm[pos["at"] % len(units)])]
                    pos["at"] += 1
                    st["n"] += 1
                c = one(u)
                with lock:
                    st["cells"] += c
        t0 = time.perf_counter()
        with ThreadPoolExecutor(cores) as ex:
            for _ in range(cores):
                ex.submit(worker)
        dt = time.perf_counter() - t0
        return {"value": st["cells"] / dt / 1e9, "unit": "Gcells/s", "cores": cores, "kind": "port",
                "sample": f"{st['n']} of {len(units)} (sequence, mode) scans of one calibration, {dt:.1f} s on "
                          f"{cores} threads (the reference runs them one after another on one core)",
                "cells": st["cells"], "seconds": dt}

    metric = "cmcalibrate scan Gcells/s (4 exp modes, bit-exact)"
    if args.impl == "reference":
        if rank != 0:
            return
        per_step = max(1.0, args.cpu_seconds / max(1, args.steps))
        for _ in range(args.warmup):
            cpu_sample(per_step)
        samples = [cpu_sample(per_step) for _ in range(args.steps)]
        cells, secs = sum(x["cells"] for x in samples), sum(x["seconds"] for x in samples)
        val = cells / secs / 1e9
        cb = {"value": val, "unit": "Gcells/s", "cores": cores, "kind": "port",
              "sample": f"{args.steps} steps of {per_step:.1f} s, each a bounded sample of one calibration's "
                        f"(sequence, mode) scans on {cores} threads"}
        print(json.dumps({"impl": "reference", "metric": metric, "value": val, "unit": "Gcells/s",
                          "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                          "ms_per_step": 1e3 * secs / max(1, args.steps), "higher_is_better": True,
                          "scaling": "weak", "vs_baseline": None, "dtype": "f32/int32", "data": "synthetic",
                          "config": config, "cpu_baseline": cb,
                          "e2e": {"value": val, "unit": "Gcells/s", "h2d_bytes_per_step": 0,
                                  "d2h_bytes_per_step": 0}}))
        return

    import torch
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(local_rank)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.int32, device="cuda")

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def call():
        return cal.calibrate_cm(cm_s, ccfg, W=W, device=local_rank)

    for _ in range(args.warmup):
        ref = call()
    clocks = ClockSampler(local_rank)
    barrier()
    clocks.start()
    walls, kms, cells, terms, launches = [], [], 0.0, 0.0, 0
    for _ in range(args.steps):
        flush.fill_(1)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        out = call()
        walls.append(1e3 * (time.perf_counter() - t0))
        kms.append(out["kernel_ms"])
        cells, terms = out["cells"], out["terms"]
        launches += out["launches"]
    barrier()
    clk = clocks.stop()
    if [e["mu"] for e in out["exp"]] != [e["mu"] for e in ref["exp"]]:
        raise RuntimeError("calibrations differ between steps")
    total_ms, e2e_ms, all_cells = aggregate_ranks(dist, sum(kms), sum(walls), cells * args.steps)
    value = all_cells / (total_ms / 1e3) / 1e9
    e2e = all_cells / (e2e_ms / 1e3) / 1e9
    sm_mhz = clk["sm_mhz"] or 1965.0
    nsm = torch.cuda.get_device_properties(local_rank).multi_processor_count
    peak = nsm * 128 * sm_mhz * 1e6 / 1e9
    # lane-ops: half the modes CYK (2 per term), half Inside (7 per term), 2 per cell
    ops = 4.5 * terms + OPS_PER_CELL * cells
    achieved = ops / (statistics.mean(kms) / 1e3) / 1e9
    cb = cpu_sample(args.cpu_seconds) if (rank == 0 and not args.no_cpu) else None
    line = {"metric": metric, "value": value, "unit": "Gcells/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": statistics.mean(walls), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32/int32", "data": "synthetic", "config": config,
            "e2e": {"value": e2e, "unit": "Gcells/s", "h2d_bytes_per_step": 4 * nseq * flen,
                    "d2h_bytes_per_step": None, "timing": "host clock around the synchronous cmgpu_calibrate call"},
            "gpu_launches": launches,
            "calibration": {"exp": out["exp"], "nhits": out["nhits"], "kernel_ms_per_step": statistics.mean(kms),
                            "wall_ms_per_step": statistics.mean(walls)},
            "roofline": {"bound": "issue", "achieved": achieved, "peak": peak, "unit": "Gop/s",
                         "frac": achieved / peak, "traffic": None,
                         "note": f"2 (CYK) / 7 (Inside) lane-ops per child term + 2 per cell; {nsm} SMs x 128 "
                                 f"lanes x {sm_mhz:.0f} MHz"},
            "cpu_baseline": cb, "clocks": clk}
    if rank == 0:
        print(json.dumps(line))
    if dist is not None:
        dist.destroy_process_group()

if __name__ == "__main__":
    main()
