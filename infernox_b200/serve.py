"""A cmscan-style serving loop: query sequences against a device-resident
library of CMs, with continuous batching.

The reference runs cmscan as a serial loop over queries and, for each, over
the models of the library (src/bin/cmscan.rs:833-834), with parallelism only
inside one search (src/cm_search.rs:1300-1315).  Here every model of the
library stays uploaded with its scan plans, all models share one device
workspace (decks and buffers sized once for the largest scan), and requests
share the GPU:

* Admission.  A submitted request waits in a bounded FIFO queue; it becomes
  active when the residues of all active requests (both strands) stay within
  the server's budget, which bounds the device memory the batched buffers and
  reportable-cell lists take.  A request larger than the whole budget, or one
  submitted to a full queue, is refused with a clear status.
* Continuous batching.  A cursor walks the library model by model, round and
  round.  Each model step scans the windows of every active request that
  still needs that model -- both strands of every query -- in one batched
  launch (cmgpu_scan_batch): the --nohmm pair of the reference for each
  window, the QDB1 CYK filter (cyk_seq_filter, src/cm_nohmm.rs:855-889) and
  then QDB2 integer Inside over its envelopes (final_stage_inside,
  src/cm_nohmm.rs:907-935), each as one launch over all requests.  A request
  admitted while the cursor stands at model k joins at model k and is done
  when the cursor has come round to k again, so it never waits for a full
  pass that started before it arrived.
* Results.  Every window is scanned exactly as it would be alone, so a
  request's hits are the same whatever else was in the batch (the test
  checks it); per model and strand they come in the reference's order.
"""
from __future__ import annotations

import collections
import time
from dataclasses import dataclass, field

import numpy as np

from . import _native as N
from .scan import CYK_F32, INSIDE_I32, QDB1, QDB2, Scanner, Workspace
from .synth import revcomp

OK, REFUSED_TOO_LARGE, REFUSED_QUEUE_FULL, CANCELLED = 0, 1, 2, 3


@dataclass
class Request:
    """One query: digital residues (codes 0..17) of the top strand."""
    rid: int
    seq: np.ndarray
    arrival: float = 0.0          # seconds on the server's clock
    status: int = OK
    admitted: float = None
    done: float = None
    start_model: int = -1          # library cursor when the request became active
    remaining: int = 0             # models still to scan
    # hits[(model, strand)] = list of (i, j, score, bias), strand 0 top / 1 bottom
    hits: dict = field(default_factory=dict)

    @property
    def residues(self) -> int:
        return 2 * int(len(self.seq))


def _pad_merge(hits, W: int, n: int):
    """cyk_seq_filter's envelopes: each hit padded by W-1 on both sides,
    clipped to [1, n], sorted by (end, start) and merged where they overlap
    (src/cm_nohmm.rs:858-888)."""
    pad = sorted(((max(1, j - (W - 1)), min(n, i + (W - 1))) for i, j in hits), key=lambda x: (x[1], x[0]))
    out = []
    k = 0
    while k < len(pad):
        s, e = pad[k]
        while k + 1 < len(pad) and pad[k + 1][0] <= e:
            k += 1
            e = max(e, pad[k][1])
        out.append((s, e))
        k += 1
    return out


def library_from_cm_file(src, local: bool = True) -> list:
    """The configured CMs of a CM file -- cmscan's CM database -- in file
    order, each keeping the W its file states (cmfile.read_cms)."""
    from . import cmfile, model
    return [model.configure(f.cm, local=local, W=f.W) for f in cmfile.read_cms(src)]


class Server:
    """The request loop over a library of configured CMs on one GPU."""

    def __init__(self, models, device: int = 0, budget_residues: int = 4_000_000, max_queue: int = 1024,
                 f6_cutoff: float = 12.0, final_cutoff: float = 15.0, do_null3: bool = True):
        self.models = list(models)
        self.device = device
        self._scanners = None  # uploaded on the first scan (queueing needs no GPU)
        self._ws = None        # one workspace shared by every model's scanner
        self.budget = int(budget_residues)
        self.max_queue = int(max_queue)
        self.f6_cutoff, self.final_cutoff, self.do_null3 = float(f6_cutoff), float(final_cutoff), bool(do_null3)
        self.queue = collections.deque()
        self.active = []
        self.finished = []
        self.cursor = 0
        self.t0 = time.perf_counter()
        self.launches = 0
        self.model_steps = 0
        self.kernel_ms = 0.0  # device time of the scans

    def clock(self) -> float:
        return time.perf_counter() - self.t0

    @property
    def scanners(self):
        if self._scanners is None:
            self._ws = Workspace(self.device)
            self._scanners = [Scanner(cm, device=self.device, workspace=self._ws) for cm in self.models]
        return self._scanners

    def close(self):
        for s in self._scanners or []:
            s.close()
        self._scanners = None
        if self._ws is not None:
            self._ws.close()
            self._ws = None

    # -- requests ----------------------------------------------------------
    def submit(self, req: Request) -> int:
        """Queue a request; returns OK or the refusal status (also stored in
        req.status).  The sequence must hold residue codes 0..17."""
        seq = np.asarray(req.seq, np.uint8)
        if seq.size and int(seq.max()) > 17:
            raise ValueError("residue code > 17 in the query")
        if req.residues > self.budget:
            req.status = REFUSED_TOO_LARGE
        elif len(self.queue) >= self.max_queue:
            req.status = REFUSED_QUEUE_FULL
        else:
            req.status = OK
            self.queue.append(req)
        return req.status

    def cancel(self, rid: int) -> bool:
        """Withdraw a queued or active request; True if it was found."""
        for coll in (self.queue, self.active):
            for r in list(coll):
                if r.rid == rid:
                    coll.remove(r)
                    r.status = CANCELLED
                    r.done = self.clock()
                    self.finished.append(r)
                    return True
        return False

    def _admit(self):
        used = sum(r.residues for r in self.active)
        while self.queue and used + self.queue[0].residues <= self.budget:
            r = self.queue.popleft()
            r.admitted = self.clock()
            r.start_model = self.cursor
            r.remaining = len(self.models)
            self.active.append(r)
            used += r.residues

    # -- one model step ----------------------------------------------------
    def step(self) -> int:
        """Admit what fits, then scan every active request against the model
        at the cursor; returns the number of requests completed."""
        self._admit()
        if not self.active:
            return 0
        k = self.cursor
        cm, sc = self.models[k], self.scanners[k]
        frames, wins, owners, off = [], [], [], 0
        for r in self.active:
            for strand, s in enumerate((r.seq, revcomp(r.seq))):
                f = np.concatenate([[255], np.asarray(s, np.uint8), [255]]).astype(np.uint8)
                frames.append(f)
                wins.append((off, 1, len(s)))
                owners.append((r, strand, len(s), off))
                off += len(f)
        buf = np.concatenate(frames)
        W = np.array(wins, dtype=N.WINDOW_DTYPE)
        # F6: QDB1 CYK over every window, one launch
        cyk = sc.scan_batch(CYK_F32, QDB1, buf, W, self.f6_cutoff, self.do_null3)
        self.launches += 1
        self.kernel_ms += sc.stats()["kernel_ms"]
        envw, env_owner = [], []
        for w, (r, strand, n, o) in enumerate(owners):
            h = cyk[cyk["win"] == w]
            for s, e in _pad_merge([(int(x["i"]), int(x["j"])) for x in h], cm.W, n):
                envw.append((o, s, e))
                env_owner.append(w)
        per_window = collections.defaultdict(list)
        if envw:
            # F7: QDB2 Inside over every envelope of every window, one launch
            E = np.array(envw, dtype=N.WINDOW_DTYPE)
            fin = sc.scan_batch(INSIDE_I32, QDB2, buf, E, self.final_cutoff, self.do_null3)
            self.launches += 1
            self.kernel_ms += sc.stats()["kernel_ms"]
            for x in fin:
                per_window[env_owner[int(x["win"])]].append(
                    (int(x["i"]), int(x["j"]), float(x["score"]), float(x["bias"])))
        for w, (r, strand, n, o) in enumerate(owners):
            r.hits[(k, strand)] = per_window.get(w, [])
        done = 0
        now = self.clock()
        for r in list(self.active):
            r.remaining -= 1
            if r.remaining == 0:
                r.done = now
                self.active.remove(r)
                self.finished.append(r)
                done += 1
        self.cursor = (k + 1) % len(self.models)
        self.model_steps += 1
        return done

    def idle(self) -> bool:
        return not self.queue and not self.active


def scan_alone(server: Server, req: Request) -> dict:
    """The hits of one request scanned on its own, model by model, through
    the same entry points (the reference's per-query loop): the check that
    batching changes nothing."""
    out = {}
    for k, (cm, sc) in enumerate(zip(server.models, server.scanners)):
        for strand, s in enumerate((req.seq, revcomp(req.seq))):
            dsq = np.concatenate([[255], np.asarray(s, np.uint8), [255]]).astype(np.uint8)
            n = len(s)
            envs = sc.cyk_seq_filter(dsq, n, server.f6_cutoff, server.do_null3)
            hits = sc.final_stage_inside(dsq, envs, server.final_cutoff, server.do_null3) if envs else []
            out[(k, strand)] = [(h.i, h.j, float(np.float32(h.score)), float(np.float32(h.bias))) for h in hits]
    return out
