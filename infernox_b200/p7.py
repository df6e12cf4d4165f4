"""P7 filter profiles and the GPU P7 filters.

Mirrors, over libcmscan_gpu.so:
  * `build_vit_filter(&P7Profile) -> VitFilter` and
    `vit_score(&VitFilter, dsq, l) -> Option<f32>` (src/p7_vitfilter.rs:121,
    :292);
  * `build_msv_filter(&P7Profile, max_length) -> MsvFilter`,
    `msv_score`, `msv_score_reconfig` and
    `f1_msv_windows(&MsvFilter, dsq, l, f1, cmw) -> Vec<Window>`
    (src/cm_pipeline.rs:201, :402, :410, :842);
  * `build_forward_filter(&P7Profile) -> ForwardFilter`,
    `build_bias_filter(&compo, m) -> BiasFilter`, `forward_filter_score`,
    `bias_filter_score` and `f3_filter_sequence` (src/cm_pipeline.rs:969,
    :1683, :1420, :1722, :1863) as FwdFilter and its functions.
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


class FwdFilter:
    """build_forward_filter(p7) and build_bias_filter(p7.compo, p7.m)
    (src/cm_pipeline.rs:969, :1683) with the local Forward exp-tail
    parameters (evparam.lftau / lflambda) of the F3 gate."""

    def __init__(self, p: P7Profile, compo, ftau: float = 0.0, flambda: float = 1.0, device: int = 0):
        self.p = p
        self._mat = np.ascontiguousarray(p.mat, np.float32).reshape(p.M + 1, 4)
        self._trans = np.ascontiguousarray(p.trans, np.float32).reshape(p.M + 1, 7)
        self._compo = np.ascontiguousarray(compo, np.float32).reshape(4)
        prof = N.P7Profile(p.M, N.ptr(self._mat, C.c_float), N.ptr(self._trans, C.c_float))
        self._h = C.c_void_p()
        N.check(N.lib().cmgpu_fwd_filter_build(C.byref(prof), self._compo.ctypes.data, float(ftau), float(flambda),
                                               device, C.byref(self._h)))

    def close(self):
        if self._h:
            N.lib().cmgpu_fwd_filter_free(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def tables(self):
        """(rfv [(M+1), 18], [(M+1), 8] = tBM, MM, IM, DM, MI, II, MD, DD, bias eo [18, 2], t1 [3])."""
        m = self.p.M
        rfv = np.zeros((m + 1, 18), np.float32)
        tr = np.zeros((m + 1, 8), np.float32)
        eo = np.zeros((18, 2), np.float32)
        t1 = np.zeros(3, np.float32)
        n = C.c_int32()
        N.check(N.lib().cmgpu_fwd_filter_tables(self._h, rfv.ctypes.data, tr.ctypes.data, m + 1, C.byref(n),
                                                eo.ctypes.data, t1.ctypes.data))
        return rfv, tr, eo, t1

    def set_kernel(self, shared: bool):
        """Force the shared-memory Forward kernel (True) or let the filter pick (False)."""
        N.check(N.lib().cmgpu_fwd_filter_set_kernel(self._h, 1 if shared else 0))

    def stats(self):
        """(kernel ms, Forward cells, launches) of the last call."""
        ms, cells, launches = C.c_double(), C.c_int64(), C.c_int32()
        N.check(N.lib().cmgpu_fwd_filter_stats(self._h, C.byref(ms), C.byref(cells), C.byref(launches)))
        return ms.value, cells.value, launches.value

    def score_batch(self, buf: np.ndarray, windows: np.ndarray, fwd: bool = True, bias: bool = True):
        """(Forward scores, bias-filter scores) in nats per window; either is
        None when not asked for."""
        b = np.ascontiguousarray(buf, np.uint8)
        w = np.ascontiguousarray(windows, N.WINDOW_DTYPE)
        fs = np.zeros(len(w), np.float32) if fwd else None
        bs = np.zeros(len(w), np.float32) if bias else None
        N.check(N.lib().cmgpu_fwd_score_batch(self._h, None, b.ctypes.data, b.size, w.ctypes.data, len(w),
                                              None if fs is None else fs.ctypes.data,
                                              None if bs is None else bs.ctypes.data))
        return fs, bs


def forward_filter_score(f: FwdFilter, dsq, l: int) -> float:
    """src/cm_pipeline.rs:1420 -- the local Forward score (nats) of dsq[1..l]."""
    return float(f.score_batch(np.ascontiguousarray(dsq, np.uint8), np.array([(0, 1, l)], N.WINDOW_DTYPE),
                               bias=False)[0][0])


def bias_filter_score(f: FwdFilter, dsq, l: int) -> float:
    """src/cm_pipeline.rs:1722 -- the composition-bias null score (nats)."""
    return float(f.score_batch(np.ascontiguousarray(dsq, np.uint8), np.array([(0, 1, l)], N.WINDOW_DTYPE),
                               fwd=False)[1][0])


def f3_filter_batch(ff: FwdFilter, buf: np.ndarray, chunks: np.ndarray, f1: float, f3: float, f3b: float, cmw: int,
                    mf: MsvFilter = None, vf: VitFilter = None, msvbias=None, vit=None, do_fwd: bool = True,
                    do_fwdbias: bool = True, do_msv: bool = True, maxw: int = 0):
    """f3_filter_sequence (src/cm_pipeline.rs:1863) on every chunk: the
    merged survivors (F1_WINDOW_DTYPE, chunk coordinates, F3b bit score) and
    the summed accounting.  msvbias = (f1b, lmmu, lmlambda) turns F1b on;
    vit = (f2, do_vitbias, f2b, lvmu, lvlambda) turns F2 / F2b on."""
    cfg = N.F3Config()
    cfg.f1, cfg.f3, cfg.f3b, cfg.cmw, cfg.maxw = float(f1), float(f3), float(f3b), int(cmw), int(maxw)
    cfg.do_msv, cfg.do_fwd, cfg.do_fwdbias = int(do_msv), int(do_fwd), int(do_fwdbias)
    cfg.f1b = cfg.f2 = cfg.f2b = 1.0
    if msvbias is not None:
        cfg.do_msvbias = 1
        cfg.f1b, cfg.lmmu, cfg.lmlambda = (float(x) for x in msvbias)
    if vit is not None:
        cfg.do_vit = 1
        f2, do_vitbias, f2b, lvmu, lvl = vit
        cfg.f2, cfg.do_vitbias, cfg.f2b, cfg.lvmu, cfg.lvlambda = float(f2), int(do_vitbias), float(f2b), \
            float(lvmu), float(lvl)
    b = np.ascontiguousarray(buf, np.uint8)
    c = np.ascontiguousarray(chunks, N.WINDOW_DTYPE)
    acct = N.F3Acct()
    cap = 1024 + b.size // 256
    while True:
        out = np.zeros(cap, F1_WINDOW_DTYPE)
        n = C.c_int32()
        rc = N.lib().cmgpu_f3_filter(ff._h, mf._h if mf is not None else None, vf._h if vf is not None else None,
                                     None, b.ctypes.data, b.size, c.ctypes.data, len(c), C.byref(cfg),
                                     out.ctypes.data, cap, C.byref(n), C.byref(acct))
        if rc == N.CMGPU_EOVERFLOW and n.value > cap:
            cap = n.value
            continue
        N.check(rc)
        return out[: n.value], {k: int(getattr(acct, k)) for k in N.F3_ACCT_FIELDS}


def f3_filter_sequence(mf: MsvFilter, ff: FwdFilter, dsq, win_len: int, f1: float, f3: float, f3b: float, cmw: int,
                       **kw):
    """src/cm_pipeline.rs:1863 on one chunk frame: ([(start, end, score)], accounting)."""
    w, acct = f3_filter_batch(ff, np.ascontiguousarray(dsq, np.uint8), np.array([(0, 1, win_len)], N.WINDOW_DTYPE),
                              f1, f3, f3b, cmw, mf=mf, **kw)
    return [(int(r["start"]), int(r["end"]), float(r["score"])) for r in w], acct


def pipeline_thresholds(z_residues: float) -> dict:
    """CmPipeline::new_default (src/cm_pipeline.rs:73-112): the filter
    thresholds and stages of the default pipeline for a database of
    z_residues residues (both strands)."""
    z_mb = z_residues / 1.0e6
    t = dict(f1=0.35, f1b=1.0, f2=1.0, f2b=1.0, f3=0.02, f3b=0.02, f4=0.02, f4b=0.02, f5=0.02, f5b=1.0, f6=0.0001,
             do_msv=True, do_msvbias=False, do_vit=True, do_vitbias=True, do_fwd=True, do_fwdbias=True)
    if z_mb >= 20000.0:
        t.update(f1=0.06, f2=0.02, f2b=0.02, f3=0.0002, f3b=0.0002, f4=0.0002, f4b=0.0002, f5=0.0002)
    elif z_mb >= 2000.0:
        t.update(f1=0.15, f2=0.15, f2b=0.15, f3=0.0002, f3b=0.0002, f4=0.0002, f4b=0.0002, f5=0.0002)
    elif z_mb >= 200.0:
        t.update(f1=0.15, f2=0.15, f2b=0.15, f3=0.0008, f3b=0.0008, f4=0.0008, f4b=0.0008, f5=0.0008)
    elif z_mb >= 20.0:
        t.update(f1=0.35, f2=0.15, f2b=0.15, f3=0.003, f3b=0.003, f4=0.003, f4b=0.003, f5=0.003)
    elif z_mb >= 2.0:
        t.update(f1=0.35, do_vit=False, do_vitbias=False, f2=1.0, f2b=1.0, f3=0.005, f3b=0.005, f4=0.005,
                 f4b=0.005, f5=0.005)
    else:
        t.update(f1=0.35, do_vit=False, do_vitbias=False, f2=1.0, f2b=1.0, f3=0.02, f3b=0.02, f4=0.02, f4b=0.02,
                 f5=0.02)
    return t


def f3_pass_for_database(ff: FwdFilter, mf: MsvFilter, vf: VitFilter, buf, chunks, z_residues: float, cmw: int,
                         lvmu: float = 0.0, lvlambda: float = 1.0):
    """The F1 -> F3b pass of the default pipeline for a database of
    z_residues residues: thresholds and stages from pipeline_thresholds (the
    Viterbi stage from 20 Mb up), then f3_filter_batch."""
    t = pipeline_thresholds(z_residues)
    vit = (t["f2"], t["do_vitbias"], t["f2b"], lvmu, lvlambda) if t["do_vit"] else None
    return f3_filter_batch(ff, buf, chunks, t["f1"], t["f3"], t["f3b"], cmw, mf=mf, vf=vf if vit else None, vit=vit,
                           do_fwd=t["do_fwd"], do_fwdbias=t["do_fwdbias"])


def mean_composition(p: P7Profile) -> np.ndarray:
    """Mean match emission over the model: the composition a synthetic
    profile's bias filter uses (profiles read from a file carry their own)."""
    return np.asarray(p.mat, np.float32)[1:].mean(axis=0).astype(np.float32)


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
