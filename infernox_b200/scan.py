"""Host-side mirror of the reference's QDB scanner entry points.

The reference exposes free functions over `&CM` (src/cm_nohmm.rs):

    cyk_seq_filter(cm, dsq, n, cutoff, do_null3) -> Vec<(i32, i32)>          :855
    final_stage_inside(cm, dsq, envs, cutoff, do_null3) -> Vec<RawHit>        :907
    final_stage_inside_opt(cm, dsq, envs, cutoff, do_null3, nonbanded)        :919
    generic_scan::<f32|i32>(cm, tab, dsq, i0, j0, cutoff, do_null3, qdbidx, nonbanded)  :406

The functions here take the same arguments (a ConfiguredCM for `&CM`, a
window-frame dsq with sentinels at 0 and n+1) and return the same values,
computed on the GPU through libcmscan_gpu.so.  Argument errors raise
ValueError, as the reference panics on them; device errors raise CmgpuError.
"""
from __future__ import annotations

import ctypes as C
from collections import namedtuple

import numpy as np

from . import _native as N
from .model import ConfiguredCM

RawHit = namedtuple("RawHit", "i j score bias")

CYK_F32, INSIDE_I32 = N.CYK_F32, N.INSIDE_I32
NOQDB, QDB1, QDB2 = N.NOQDB, N.QDB1, N.QDB2
KERNEL_AUTO, KERNEL_LEVEL, KERNEL_SWEEP = N.KERNEL_AUTO, N.KERNEL_LEVEL, N.KERNEL_SWEEP
SMX_QDB1_TIGHT, SMX_QDB2_LOOSE = QDB1, QDB2


def _frame(dsq) -> np.ndarray:
    a = np.ascontiguousarray(dsq, dtype=np.uint8)
    if a.ndim != 1 or a.size < 2 or a[0] != 255 or a[-1] != 255:
        raise ValueError("dsq must be a window frame [255, residues.., 255]")
    if a.size > 2 and int(a[1:-1].max()) > 17:
        raise ValueError("residue codes must be 0..17")
    return a


class Workspace:
    """A device workspace (decks, work queue, candidate buffers, stream) that
    several Scanners of one thread may share, so a library of models keeps
    one set of scratch buffers sized for the largest scan instead of one per
    model."""

    def __init__(self, device: int = 0, stream: int | None = None):
        self.handle = C.c_void_p()
        N.check(N.lib().cmgpu_workspace_create(device, C.c_void_p(stream) if stream else None,
                                               C.byref(self.handle)))

    def close(self) -> None:
        if self.handle:
            N.lib().cmgpu_workspace_free(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Scanner:
    """A configured CM uploaded to one GPU, with a private workspace or a
    shared one (`workspace`, owned by the caller).

    One Scanner -- and one Workspace -- must be used by one thread at a time;
    build one per thread (the device model is read-only and cheap to
    re-upload)."""

    def __init__(self, cm: ConfiguredCM, device: int = 0, stream: int | None = None,
                 workspace: Workspace | None = None):
        L = N.lib()
        self.cm = cm
        self._model = C.c_void_p()
        N.check(L.cmgpu_model_upload(C.byref(cm.as_struct()), device, C.byref(self._model)))
        self._shared = workspace
        if workspace is not None:
            self._ws = workspace.handle
        else:
            self._ws = C.c_void_p()
            N.check(L.cmgpu_workspace_create(device, C.c_void_p(stream) if stream else None,
                                             C.byref(self._ws)))

    def close(self) -> None:
        L = N.lib()
        if self._ws:
            if self._shared is None:
                L.cmgpu_workspace_free(self._ws)
            self._ws = C.c_void_p()
        if self._model:
            L.cmgpu_model_free(self._model)
            self._model = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_shape(self, ctas_per_sm: int = 0, threads: int = 0, chunk: int = 0, lanes: int = 0) -> None:
        N.check(N.lib().cmgpu_workspace_set_shape(self._ws, ctas_per_sm, threads, chunk, lanes))

    def set_kernel(self, kernel: int) -> None:
        """KERNEL_AUTO, KERNEL_LEVEL (CTA level schedule) or KERNEL_SWEEP (warp node sweep)."""
        N.check(N.lib().cmgpu_workspace_set_kernel(self._ws, kernel))

    def autotune(self, semiring: int, qdbidx: int, buf: np.ndarray, windows: np.ndarray,
                 cutoff: float, device_buf=None, lanes=(4, 8, 16), threads=(512,), chunks_w=(0, 4, 8, 16)) -> dict:
        """Pick the launch shape (work items per CTA, threads per CTA) and the
        work-item length (0 = automatic, else that many multiples of W: longer
        pieces repeat fewer W-1 warm-up columns, shorter ones balance the
        tail) for this model and batch by timing one scan per candidate; the
        fastest stays set on this Scanner.  Every candidate returns the same
        hits (checked)."""
        best, ref, trials = None, None, []
        for th in threads:
            for ln in lanes:
                for cw in chunks_w:
                    chunk = int(cw * self.cm.W)
                    self.set_shape(0, th, chunk, ln)
                    hits = self.scan_batch(semiring, qdbidx, buf, windows, cutoff, False, device_buf=device_buf)
                    ms = self.stats()["kernel_ms"]
                    if ref is None:
                        ref = hits
                    elif not np.array_equal(hits, ref):
                        raise RuntimeError("launch shapes disagree")
                    trials.append({"lanes": ln, "threads": th, "chunk": chunk, "kernel_ms": ms})
                    if best is None or ms < best["kernel_ms"]:
                        best = trials[-1]
        self.set_shape(0, best["threads"], best["chunk"], best["lanes"])
        return {"best": best, "trials": trials}

    def stats(self) -> dict:
        s = N.Stats()
        N.check(N.lib().cmgpu_workspace_stats(self._ws, C.byref(s)))
        return {k: getattr(s, k) for k, _ in N.Stats._fields_}

    # ------------------------------------------------------------------
    def generic_scan(self, semiring: int, qdbidx: int, dsq, i0: int, j0: int, cutoff: float,
                     do_null3: bool) -> list:
        a = _frame(dsq)
        n = a.size - 2
        if not (1 <= i0 and j0 <= n):
            raise ValueError("window outside the frame")
        cap = max(64, (j0 - i0 + 1) // 4 + 64)
        while True:
            out = np.zeros(cap, N.HIT_DTYPE)
            nout = C.c_int32()
            rc = N.lib().cmgpu_qdb_scan(self._model, self._ws, semiring, qdbidx,
                                        N.ptr(a, C.c_uint8), n, i0, j0, float(cutoff),
                                        int(bool(do_null3)), out.ctypes.data, cap, C.byref(nout))
            if rc == N.CMGPU_EOVERFLOW:
                cap = nout.value + 16
                continue
            N.check(rc)
            return [RawHit(int(h["i"]), int(h["j"]), float(h["score"]), float(h["bias"]))
                    for h in out[: nout.value]]

    def scan_cells(self, semiring: int, qdbidx: int, dsq, i0: int, j0: int, cutoff: float):
        """Reportable cells (j, d, bits) of a window scan, sorted by (j, d)."""
        a = _frame(dsq)
        n = a.size - 2
        cap = max(1024, (j0 - i0 + 1) * (self.cm.W + 2))
        cj = np.zeros(cap, np.int32)
        cd = np.zeros(cap, np.int32)
        cs = np.zeros(cap, np.float32)
        nout = C.c_int32()
        N.check(N.lib().cmgpu_qdb_scan_cells(self._model, self._ws, semiring, qdbidx,
                                             N.ptr(a, C.c_uint8), n, i0, j0, float(cutoff),
                                             cj.ctypes.data, cd.ctypes.data, cs.ctypes.data, cap,
                                             C.byref(nout)))
        k = nout.value
        return list(zip(cj[:k].tolist(), cd[:k].tolist(), cs[:k].tolist()))

    def cyk_seq_filter(self, dsq, n: int, cutoff: float, do_null3: bool) -> list:
        a = _frame(dsq)
        if n != a.size - 2:
            raise ValueError("n must equal the frame length")
        cap = 1024
        while True:
            out = np.zeros(cap, N.ENV_DTYPE)
            nout = C.c_int32()
            rc = N.lib().cmgpu_cyk_seq_filter(self._model, self._ws, N.ptr(a, C.c_uint8), n,
                                              float(cutoff), int(bool(do_null3)), out.ctypes.data,
                                              cap, C.byref(nout))
            if rc == N.CMGPU_EOVERFLOW:
                cap = nout.value + 16
                continue
            N.check(rc)
            return [(int(e["start"]), int(e["end"])) for e in out[: nout.value]]

    def final_stage_inside_opt(self, dsq, envs, cutoff: float, do_null3: bool,
                               nonbanded: bool) -> list:
        a = _frame(dsq)
        n = a.size - 2
        ev = np.asarray([tuple(e) for e in envs], N.ENV_DTYPE) if len(envs) else np.zeros(0, N.ENV_DTYPE)
        cap = max(64, 16 * len(ev))
        while True:
            out = np.zeros(cap, N.HIT_DTYPE)
            nout = C.c_int32()
            rc = N.lib().cmgpu_final_stage_inside_opt(
                self._model, self._ws, N.ptr(a, C.c_uint8), n, ev.ctypes.data, len(ev),
                float(cutoff), int(bool(do_null3)), int(bool(nonbanded)), out.ctypes.data, cap,
                C.byref(nout))
            if rc == N.CMGPU_EOVERFLOW:
                cap = nout.value + 16
                continue
            N.check(rc)
            return [RawHit(int(h["i"]), int(h["j"]), float(h["score"]), float(h["bias"]))
                    for h in out[: nout.value]]

    def final_stage_inside(self, dsq, envs, cutoff: float, do_null3: bool) -> list:
        return self.final_stage_inside_opt(dsq, envs, cutoff, do_null3, False)

    # ------------------------------------------------------------------
    def calibrate_scan_batch(self, semiring: int, qdbidx: int, buf: np.ndarray, windows: np.ndarray,
                             do_null3: bool) -> np.ndarray:
        """cmcalibrate's scan of every window (cutoff -inf, local begins in
        bit-score order, src/cm_calibrate.rs:441-989): the kept hits of each
        window, BATCH_HIT_DTYPE in window order."""
        w = np.ascontiguousarray(windows, N.WINDOW_DTYPE)
        b = np.ascontiguousarray(buf, np.uint8)
        # kept hits of a window are disjoint: at most one per residue
        cap = max(1024, int((w["j0"] - w["i0"] + 1).clip(0).sum()) + len(w))
        out = np.zeros(cap, N.BATCH_HIT_DTYPE)
        nout = C.c_int32()
        N.check(N.lib().cmgpu_calibrate_scan_batch(self._model, self._ws, semiring, qdbidx, b.ctypes.data,
                                                   int(b.size), w.ctypes.data, len(w), int(bool(do_null3)),
                                                   out.ctypes.data, cap, C.byref(nout)))
        return out[: nout.value].copy()

    def scan_batch(self, semiring: int, qdbidx: int, buf: np.ndarray, windows: np.ndarray,
                   cutoff: float, do_null3: bool, plain: bool = False, device_buf=None) -> np.ndarray:
        """Scan many windows of one residue buffer in one launch.

        buf: uint8 buffer of concatenated window frames; windows: WINDOW_DTYPE
        array.  device_buf: optional device pointer (int) to a resident copy
        of buf (then buf is not copied).  Returns BATCH_HIT_DTYPE hits grouped
        by window in window order."""
        w = np.ascontiguousarray(windows, N.WINDOW_DTYPE)
        cap = max(1024, len(w) * 4)
        L = N.lib()
        while True:
            out = np.zeros(cap, N.BATCH_HIT_DTYPE)
            nout = C.c_int32()
            if device_buf is not None:
                rc = L.cmgpu_scan_batch_device(self._model, self._ws, semiring, qdbidx,
                                               C.c_void_p(device_buf), int(buf.size), w.ctypes.data,
                                               len(w), float(cutoff), int(bool(do_null3)),
                                               out.ctypes.data, cap, C.byref(nout))
            else:
                b = np.ascontiguousarray(buf, np.uint8)
                fn = L.cmgpu_scan_plain if plain else L.cmgpu_scan_batch
                rc = fn(self._model, self._ws, semiring, qdbidx, N.ptr(b, C.c_uint8), int(b.size),
                        w.ctypes.data, len(w), float(cutoff), int(bool(do_null3)), out.ctypes.data,
                        cap, C.byref(nout))
            if rc == N.CMGPU_EOVERFLOW:
                cap = nout.value + 16
                continue
            N.check(rc)
            return out[: nout.value].copy()


_scanners: dict = {}


def _scanner(cm: ConfiguredCM) -> Scanner:
    s = _scanners.get(id(cm))
    if s is None or s.cm is not cm:
        s = Scanner(cm)
        _scanners[id(cm)] = s
    return s


def cyk_seq_filter(cm: ConfiguredCM, dsq, n: int, cutoff: float, do_null3: bool) -> list:
    """src/cm_nohmm.rs:855 -- envelopes (start, end) of the QDB1 CYK filter."""
    return _scanner(cm).cyk_seq_filter(dsq, n, cutoff, do_null3)


def final_stage_inside(cm: ConfiguredCM, dsq, envs, cutoff: float, do_null3: bool) -> list:
    """src/cm_nohmm.rs:907 -- QDB2 integer Inside hits over the envelopes."""
    return _scanner(cm).final_stage_inside_opt(dsq, envs, cutoff, do_null3, False)


def final_stage_inside_opt(cm: ConfiguredCM, dsq, envs, cutoff: float, do_null3: bool,
                           nonbanded: bool) -> list:
    """src/cm_nohmm.rs:919 -- as final_stage_inside; nonbanded selects the full d-range."""
    return _scanner(cm).final_stage_inside_opt(dsq, envs, cutoff, do_null3, nonbanded)


def generic_scan(cm: ConfiguredCM, semiring: int, dsq, i0: int, j0: int, cutoff: float,
                 do_null3: bool, qdbidx: int, nonbanded: bool = False) -> list:
    """src/cm_nohmm.rs:406 -- one window scan, hits after overlap removal."""
    return _scanner(cm).generic_scan(semiring, NOQDB if nonbanded else qdbidx, dsq, i0, j0,
                                     cutoff, do_null3)
