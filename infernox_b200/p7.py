"""P7 filter profiles and the GPU P7 filters.

Mirrors, over libcmscan_gpu.so:
  * `build_vit_filter(&P7Profile) -> VitFilter` and
    `vit_score(&VitFilter, dsq, l) -> Option<f32>` (src/p7_vitfilter.rs:121,
    :292);
  * `build_msv_filter(&P7Profile, max_length) -> MsvFilter`,
    `msv_score`, `msv_score_reconfig` and
    `f1_msv_windows(&MsvFilter, dsq, l, f1, cmw) -> Vec<Window>`
    (src/cm_pipeline.rs:201, :402, :410, :842).
The batch methods score or scan many windows / chunks in one call.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _native as N


@dataclass
class P7Profile:
    """Match emissions mat[0..M][4] (row 0 unused) and transitions
    trans[0..M][7] = MM, MI, MD, IM, II, DM, DD (src/p7_hmm.rs:62-92)."""
    M: int
    mat: np.ndarray
    trans: np.ndarray


class VitFilter:
    def __init__(self, p: P7Profile, device: int = 0):
        self.p = p
        self._mat = np.ascontiguousarray(p.mat, np.float32).reshape(p.M + 1, 4)
        self._trans = np.ascontiguousarray(p.trans, np.float32).reshape(p.M + 1, 7)
        prof = N.P7Profile(p.M, N.ptr(self._mat, C.c_float), N.ptr(self._trans, C.c_float))
        self._h = C.c_void_p()
        N.check(N.lib().cmgpu_vit_filter_build(C.byref(prof), device, C.byref(self._h)))

    def close(self):
        if self._h:
            N.lib().cmgpu_vit_filter_free(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def tables(self):
        n = C.c_int32()
        sp = np.zeros(3, np.int16)
        N.lib().cmgpu_vit_filter_tables(self._h, None, 0, C.byref(n), None)
        tab = np.zeros(n.value, np.int16)
        N.check(N.lib().cmgpu_vit_filter_tables(self._h, tab.ctypes.data, n.value, C.byref(n), sp.ctypes.data))
        return tab, sp

    def score_batch(self, buf: np.ndarray, windows: np.ndarray):
        """Scores (f32 bits) and scored flags (0 = None, overflow) per window."""
        b = np.ascontiguousarray(buf, np.uint8)
        w = np.ascontiguousarray(windows, N.WINDOW_DTYPE)
        sc = np.zeros(len(w), np.float32)
        ok = np.zeros(len(w), np.uint8)
        N.check(N.lib().cmgpu_vit_score_batch(self._h, None, b.ctypes.data, b.size, w.ctypes.data, len(w),
                                              sc.ctypes.data, ok.ctypes.data))
        return sc, ok


def vit_stats(f: VitFilter):
    """(kernel ms, cells, launches) of the last score_batch call."""
    ms, cells, launches = C.c_double(), C.c_int64(), C.c_int32()
    N.check(N.lib().cmgpu_vit_filter_stats(f._h, C.byref(ms), C.byref(cells), C.byref(launches)))
    return ms.value, cells.value, launches.value


def vit_score(f: VitFilter, dsq, l: int):
    """src/p7_vitfilter.rs:292 -- Some(score) or None."""
    a = np.ascontiguousarray(dsq, np.uint8)
    w = np.array([(0, 1, l)], N.WINDOW_DTYPE)
    sc, ok = f.score_batch(a, w)
    return float(sc[0]) if ok[0] else None


F1_WINDOW_DTYPE = np.dtype([("start", np.int64), ("end", np.int64), ("score", np.float32), ("chunk", np.int32)])
SSV_DIAG_DTYPE = np.dtype([("n", np.int64), ("length", np.int64), ("k", np.int64), ("score", np.float32),
                           ("chunk", np.int32)])


class MsvFilter:
    """build_msv_filter(p7, max_length) plus the profile's local MSV Gumbel
    parameters (evparam.lmmu / lmlambda), which the SSV threshold needs."""

    def __init__(self, p: P7Profile, max_length: int, lmmu: float = 0.0, lmlambda: float = 1.0, device: int = 0):
        self.p = p
        self.max_length = int(max_length)
        self._mat = np.ascontiguousarray(p.mat, np.float32).reshape(p.M + 1, 4)
        self._trans = np.ascontiguousarray(p.trans, np.float32).reshape(p.M + 1, 7)
        prof = N.P7Profile(p.M, N.ptr(self._mat, C.c_float), N.ptr(self._trans, C.c_float))
        self._h = C.c_void_p()
        N.check(N.lib().cmgpu_msv_filter_build(C.byref(prof), self.max_length, float(lmmu), float(lmlambda), device,
                                               C.byref(self._h)))

    def close(self):
        if self._h:
            N.lib().cmgpu_msv_filter_free(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def tables(self):
        """(rbv [(M+1)*18] u8, [base, bias, tbm, tec, tjb], prefix, suffix, scale_b)."""
        n = C.c_int32()
        m = self.p.M
        b5 = np.zeros(5, np.uint8)
        pre = np.zeros(m + 1, np.float32)
        suf = np.zeros(m + 1, np.float32)
        sc = C.c_float()
        N.lib().cmgpu_msv_filter_tables(self._h, None, 0, C.byref(n), None, None, None, None)
        rbv = np.zeros(n.value, np.uint8)
        N.check(N.lib().cmgpu_msv_filter_tables(self._h, rbv.ctypes.data, n.value, C.byref(n), b5.ctypes.data,
                                                pre.ctypes.data, suf.ctypes.data, C.byref(sc)))
        return rbv, b5, pre, suf, np.float32(sc.value)

    def threshold(self, f1: float) -> int:
        t = C.c_int32()
        N.check(N.lib().cmgpu_ssv_threshold(self._h, float(f1), C.byref(t)))
        return t.value

    def stats(self):
        ms, cells, launches = C.c_double(), C.c_int64(), C.c_int32()
        N.check(N.lib().cmgpu_msv_filter_stats(self._h, C.byref(ms), C.byref(cells), C.byref(launches)))
        return ms.value, cells.value, launches.value

    def score_batch(self, buf: np.ndarray, windows: np.ndarray, wlen=None):
        """msv_score (wlen None) or msv_score_reconfig per window: (scores f32, scored u8; 0 = None)."""
        b = np.ascontiguousarray(buf, np.uint8)
        w = np.ascontiguousarray(windows, N.WINDOW_DTYPE)
        wl = None if wlen is None else np.ascontiguousarray(wlen, np.int32)
        sc = np.zeros(len(w), np.float32)
        ok = np.zeros(len(w), np.uint8)
        N.check(N.lib().cmgpu_msv_score_batch(self._h, None, b.ctypes.data, b.size, w.ctypes.data, len(w),
                                              None if wl is None else wl.ctypes.data, sc.ctypes.data,
                                              ok.ctypes.data))
        return sc, ok

    def _grow(self, fn, dtype, *args, cap=256):
        while True:
            out = np.zeros(cap, dtype)
            n = C.c_int32()
            rc = fn(*args, out.ctypes.data, cap, C.byref(n))
            if rc == N.CMGPU_EOVERFLOW and n.value > cap:
                cap = n.value
                continue
            N.check(rc)
            return out[: n.value]

    def f1_windows_batch(self, buf: np.ndarray, chunks: np.ndarray, f1: float, cmw: int) -> np.ndarray:
        """f1_msv_windows on every chunk: F1_WINDOW_DTYPE rows grouped by chunk."""
        b = np.ascontiguousarray(buf, np.uint8)
        c = np.ascontiguousarray(chunks, N.WINDOW_DTYPE)
        return self._grow(N.lib().cmgpu_f1_msv_windows, F1_WINDOW_DTYPE, self._h, None, b.ctypes.data, b.size,
                          c.ctypes.data, len(c), float(f1), int(cmw), cap=4096 + b.size // 64)

    def ssv_diagonals_batch(self, buf: np.ndarray, chunks: np.ndarray, f1: float) -> np.ndarray:
        b = np.ascontiguousarray(buf, np.uint8)
        c = np.ascontiguousarray(chunks, N.WINDOW_DTYPE)
        return self._grow(N.lib().cmgpu_ssv_diagonals, SSV_DIAG_DTYPE, self._h, None, b.ctypes.data, b.size,
                          c.ctypes.data, len(c), float(f1), cap=4096 + b.size // 64)


def msv_score(f: MsvFilter, dsq, l: int):
    """src/cm_pipeline.rs:402 -- Some(score) or None."""
    sc, ok = f.score_batch(np.ascontiguousarray(dsq, np.uint8), np.array([(0, 1, l)], N.WINDOW_DTYPE))
    return float(sc[0]) if ok[0] else None


def msv_score_reconfig(f: MsvFilter, dsq, l: int, wlen: int):
    """src/cm_pipeline.rs:410 -- the MSV score with the length model set to wlen."""
    sc, ok = f.score_batch(np.ascontiguousarray(dsq, np.uint8), np.array([(0, 1, l)], N.WINDOW_DTYPE), [wlen])
    return float(sc[0]) if ok[0] else None


def f1_msv_windows(f: MsvFilter, dsq, l: int, f1: float, cmw: int):
    """src/cm_pipeline.rs:842 -- [(start, end, score)] of one chunk frame."""
    w = f.f1_windows_batch(np.ascontiguousarray(dsq, np.uint8), np.array([(0, 1, l)], N.WINDOW_DTYPE), f1, cmw)
    return [(int(r["start"]), int(r["end"]), float(r["score"])) for r in w]


def synthetic_profile(m: int, seed: int, peak: float = 0.6):
    """A seeded p7 filter profile: one preferred residue per match state with
    probability `peak`, insert/delete transitions of a few percent.  Returns
    the profile and its consensus residues (index k = 1..M)."""
    r = np.random.default_rng(seed)
    mat = np.zeros((m + 1, 4), np.float32)
    cons = r.integers(0, 4, m + 1)
    for k in range(1, m + 1):
        v = r.uniform(0.5, 1.5, 4)
        v[cons[k]] = 0.0
        v = v / v.sum() * (1.0 - peak)
        v[cons[k]] = peak
        mat[k] = v.astype(np.float32)
    trans = np.zeros((m + 1, 7), np.float32)
    for k in range(m + 1):
        mi, md = r.uniform(0.01, 0.05, 2)
        ii, dd = r.uniform(0.2, 0.5), r.uniform(0.2, 0.5)
        trans[k] = [1 - mi - md, mi, md, 1 - ii, ii, 1 - dd, dd]
    return P7Profile(m, mat, trans), cons


def planted_residues(n: int, cons, nplant: int, seed: int, mut: float = 0.25, gc: float = 0.5) -> np.ndarray:
    """n i.i.d. residue codes (0..3) with nplant mutated consensus runs."""
    r = np.random.default_rng(seed)
    p = np.array([(1 - gc) / 2, gc / 2, gc / 2, (1 - gc) / 2])
    seq = r.choice(4, n, p=p).astype(np.uint8)
    m = len(cons) - 1
    for _ in range(nplant):
        run = np.array(cons[1:], np.uint8)
        flip = r.random(m) < mut
        run[flip] = r.integers(0, 4, int(flip.sum()))
        if m < n:
            q = int(r.integers(0, n - m))
            seq[q:q + m] = run
    return seq
