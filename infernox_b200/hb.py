"""HMM-banded (CP9-banded) scanners on the GPU.

Mirrors the reference's functions over `&CM` and `&CP9Bands`
(src/cp9.rs):

    fast_cyk_scan_hb(cm, cp9b, dsq, i0, j0, env_cutoff) -> (vsc_root, envi, envj)       :4682
    fast_fcyk_scan_hb(cm, cp9b, dsq, i0, j0, env_cutoff, cutoff, do_null3)
        -> (vsc_root, envi, envj, hits)                                                 :4704
    fast_finside_scan_hb(cm, cp9b, dsq, i0, j0, env_cutoff, cutoff, do_null3)
        -> (vsc_root, envi, envj, hits)                                                 :5465

and the truncated scanners (src/cm_dpsearch_trunc.rs):

    tr_cyk_scan_hb(cm, trp, cp9b, dsq, i0, j0, cutoff, do_null3, pass_idx, env_cutoff, local)
        -> (hits, vsc_root, vmode_root, envi, envj)                                     :264
    ftr_inside_scan_hb(...) (same)                                                      :1055

`Bands` holds what the scanners read from CP9Bands: jmin/jmax per state and
the per-row d-bands hdmin/hdmax (and, for the truncated scans, the per-state
J/L/R/T validity).  `TrInputs` holds what the truncated scanners select from
the CM and TrPenalties for one pass.  The batch functions scan many
envelopes, each with its own bands, in one call.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _native as N
from .scan import Scanner, _frame, _scanner


@dataclass
class Bands:
    """jmin/jmax [M]; hdmin/hdmax rows of state v at hd_off[v] + (j - jmin[v])."""
    jmin: np.ndarray
    jmax: np.ndarray
    hd_off: np.ndarray
    hdmin: np.ndarray
    hdmax: np.ndarray

    @staticmethod
    def from_rows(jmin, jmax, rows_min, rows_max) -> "Bands":
        """Build from per-state row lists (hdmin[v][jp], hdmax[v][jp]) as CP9Bands stores them."""
        off, acc = [], 0
        for r in rows_min:
            off.append(acc)
            acc += len(r)
        cat = lambda rs: np.ascontiguousarray(np.concatenate([np.asarray(r, np.int32) for r in rs] or [np.zeros(0)]),
                                              np.int32)
        return Bands(np.ascontiguousarray(jmin, np.int32), np.ascontiguousarray(jmax, np.int32),
                     np.asarray(off, np.int32), cat(rows_min), cat(rows_max))

    def _arrays(self):
        k = getattr(self, "_keep", None)
        if k is None or any(a is not b for a, b in zip(k[1], (self.jmin, self.jmax, self.hd_off, self.hdmin,
                                                             self.hdmax))):
            src = (self.jmin, self.jmax, self.hd_off, self.hdmin, self.hdmax)
            arrs = [np.ascontiguousarray(a, np.int32) for a in src]
            self._keep = k = (arrs, src, [a.ctypes.data for a in arrs])
        return k

    def pointers(self):
        """Data addresses of jmin, jmax, hd_off, hdmin, hdmax (int32, contiguous), kept alive by self."""
        return self._arrays()[2]

    def struct(self) -> N.HbBands:
        ip = lambda a: a.ctypes.data_as(C.POINTER(C.c_int32))
        return N.HbBands(*[ip(a) for a in self._arrays()[0]])


_E_ST = 7


def _sdelta(st: int) -> int:
    return 2 if st == 1 else (1 if st in (2, 3, 4, 5) else 0)


def ij2d_bands(sttype, imin, imax, jmin, jmax) -> Bands:
    """ij2d_bands (src/cp9.rs:3815-3850, non-truncated): per-state i/j bands
    to d-bands.  END rows are 0..0; other rows hdmin = max(j - imax + 1, sd),
    hdmax = j - imin + 1, empty (-1/-2) when hdmax < sd."""
    mins, maxs = [], []
    for v, st in enumerate(np.asarray(sttype)):
        st = int(st)
        n = max(0, int(jmax[v]) - int(jmin[v]) + 1)
        j = np.arange(int(jmin[v]), int(jmin[v]) + n, dtype=np.int64)
        if st == _E_ST:
            mins.append(np.zeros(n, np.int32))
            maxs.append(np.zeros(n, np.int32))
            continue
        dn = _sdelta(st)
        hdn = j - int(imax[v]) + 1
        hdx = j - int(imin[v]) + 1
        mins.append(np.where(hdx < dn, -1, np.maximum(hdn, dn)).astype(np.int32))
        maxs.append(np.where(hdx < dn, -2, hdx).astype(np.int32))
    return Bands.from_rows(jmin, jmax, mins, maxs)


def _hits(arr, n):
    return [(int(h["i"]), int(h["j"]), float(h["score"]), float(h["bias"])) for h in arr[:n]]


def _hb_hits(sc: Scanner, semiring, bands: Bands, dsq, i0, j0, env_cutoff, cutoff, do_null3):
    a = _frame(dsq)
    b = bands.struct()
    vsc, ei, ej = C.c_float(), C.c_int64(), C.c_int64()
    cap = 256
    while True:
        out = np.zeros(cap, N.HIT_DTYPE)
        n = C.c_int32()
        rc = N.lib().cmgpu_hb_scan_hits(sc._model, semiring, C.byref(b), a.ctypes.data, a.size - 2, i0, j0,
                                        float(env_cutoff), float(cutoff), int(bool(do_null3)), C.byref(vsc),
                                        C.byref(ei), C.byref(ej), out.ctypes.data, cap, C.byref(n))
        if rc == N.CMGPU_EOVERFLOW and n.value > cap:
            cap = n.value
            continue
        N.check(rc)
        return vsc.value, ei.value, ej.value, _hits(out, n.value)


def fast_cyk_scan_hb(cm, bands: Bands, dsq, i0: int, j0: int, env_cutoff: float):
    """src/cp9.rs:4682 -- (vsc_root, envi, envj); envi/envj -1 when no cell reaches env_cutoff."""
    sc = cm if isinstance(cm, Scanner) else _scanner(cm)
    a = _frame(dsq)
    b = bands.struct()
    vsc, ei, ej = C.c_float(), C.c_int64(), C.c_int64()
    N.check(N.lib().cmgpu_fast_cyk_scan_hb(sc._model, C.byref(b), a.ctypes.data, a.size - 2, i0, j0,
                                           float(env_cutoff), C.byref(vsc), C.byref(ei), C.byref(ej)))
    return vsc.value, ei.value, ej.value


def fast_fcyk_scan_hb(cm, bands: Bands, dsq, i0: int, j0: int, env_cutoff: float, cutoff: float, do_null3: bool):
    """src/cp9.rs:4704 -- (vsc_root, envi, envj, hits (i, j, score, bias) before overlap removal)."""
    sc = cm if isinstance(cm, Scanner) else _scanner(cm)
    return _hb_hits(sc, N.CYK_F32, bands, dsq, i0, j0, env_cutoff, cutoff, do_null3)


def fast_finside_scan_hb(cm, bands: Bands, dsq, i0: int, j0: int, env_cutoff: float, cutoff: float,
                         do_null3: bool):
    """src/cp9.rs:5465 -- float Inside (FLogsum); same returns as fast_fcyk_scan_hb."""
    sc = cm if isinstance(cm, Scanner) else _scanner(cm)
    return _hb_hits(sc, N.INSIDE_F32, bands, dsq, i0, j0, env_cutoff, cutoff, do_null3)


def _task_array(tasks, nvalid):
    """The tasks as an array laid out like cmgpu_hb_task (nvalid = 0) or
    cmgpu_tr_task (nvalid = 4 validity pointers), filled column by column."""
    names = ["dsq_offset", "i0", "j0", "env_cutoff", "cutoff", "p"]
    fmts = [np.int64, np.int32, np.int32, np.float32, np.float32, (np.uint64, 5 + nvalid)]
    dt = np.dtype({"names": names, "formats": fmts, "offsets": [0, 8, 12, 16, 20, 24],
                   "itemsize": 24 + 8 * (5 + nvalid)})
    a = np.zeros(len(tasks), dt)
    if not len(tasks):
        return a
    cols = list(zip(*[t[:5] for t in tasks]))
    for name, col in zip(names[:5], cols):
        a[name] = col
    a["p"][:, :5] = [t[5].pointers() for t in tasks]
    return a


def _results(res, dt):
    return np.frombuffer(res, dt) if len(res) else np.zeros(0, dt)


_HB_RES_DTYPE = np.dtype({"names": ["vsc_root", "nhits", "envi", "envj", "hit_first"],
                          "formats": [np.float32, np.int32, np.int64, np.int64, np.int64],
                          "offsets": [0, 4, 8, 16, 24], "itemsize": 32})


def hb_scan_batch(sc: Scanner, semiring: int, report_hits: bool, do_null3: bool, buf: np.ndarray, tasks):
    """tasks: [(dsq_offset, i0, j0, env_cutoff, cutoff, Bands)] -> [(vsc, envi, envj, hits)] per task."""
    b = np.ascontiguousarray(buf, np.uint8)
    tk = _task_array(tasks, 0)
    assert tk.dtype.itemsize == C.sizeof(N.HbTask)
    res = (N.HbResult * max(len(tasks), 1))()
    cap = 1024 + 16 * len(tasks)
    while True:
        out = np.zeros(cap, N.HIT_DTYPE)
        n = C.c_int64()
        rc = N.lib().cmgpu_hb_scan_batch(sc._model, None, semiring, int(bool(report_hits)), int(bool(do_null3)),
                                         b.ctypes.data, b.size, tk.ctypes.data, len(tasks), res, out.ctypes.data,
                                         cap, C.byref(n))
        if rc == N.CMGPU_EOVERFLOW and n.value > cap:
            cap = n.value
            continue
        N.check(rc)
        r = _results(res, _HB_RES_DTYPE)[:len(tasks)]
        hl = out[:n.value].tolist()
        return [(float(v), int(ei), int(ej), hl[f:f + h]) for v, h, ei, ej, f in r.tolist()]


def hb_stats(sc: Scanner):
    ms, cells, launches = C.c_double(), C.c_int64(), C.c_int32()
    N.check(N.lib().cmgpu_hb_stats(sc._model, C.byref(ms), C.byref(cells), C.byref(launches)))
    return ms.value, cells.value, launches.value


@dataclass
class TrInputs:
    """Per-pass inputs of the truncated scanners: lmesc/rmesc [M*18], the
    pass's truncated-begin penalties pty [M], the node spans lpos/rpos [M]
    that allow_truncation reads, clen, and whether local rules apply; the
    integer tables ilmesc/irmesc/ipty for the integer Inside scan."""
    lmesc: np.ndarray
    rmesc: np.ndarray
    pty: np.ndarray
    lpos: np.ndarray
    rpos: np.ndarray
    clen: int
    local: bool
    ilmesc: np.ndarray = None
    irmesc: np.ndarray = None
    ipty: np.ndarray = None

    def struct(self) -> N.TrTables:
        self._keep = [np.ascontiguousarray(self.lmesc, np.float32), np.ascontiguousarray(self.rmesc, np.float32),
                      np.ascontiguousarray(self.pty, np.float32), np.ascontiguousarray(self.lpos, np.int32),
                      np.ascontiguousarray(self.rpos, np.int32)]
        fp = lambda a: a.ctypes.data_as(C.POINTER(C.c_float))
        ip = lambda a: a.ctypes.data_as(C.POINTER(C.c_int32))
        k = self._keep
        ints = [None if x is None else np.ascontiguousarray(x, np.int32) for x in (self.ilmesc, self.irmesc, self.ipty)]
        k.extend(ints)
        ipn = lambda a: None if a is None else ip(a)
        return N.TrTables(fp(k[0]), fp(k[1]), fp(k[2]), ip(k[3]), ip(k[4]), int(self.clen), int(bool(self.local)),
                          ipn(ints[0]), ipn(ints[1]), ipn(ints[2]))


def _tr_hits(arr, n):
    return [(int(h["i"]), int(h["j"]), float(h["score"]), float(h["bias"]), int(h["mode"]), int(h["root"]))
            for h in arr[:n]]


def _u8p(a):
    return a.ctypes.data_as(C.POINTER(C.c_uint8))


def _tr_scan(sc, semiring, tri: TrInputs, bands: Bands, valid, dsq, i0, j0, cutoff, do_null3, pass_idx, env_cutoff):
    a = _frame(dsq)
    b = bands.struct()
    tt = tri.struct()
    vs = [np.ascontiguousarray(x, np.uint8) for x in valid]
    vsc, vmode, ei, ej = C.c_float(), C.c_int32(), C.c_int64(), C.c_int64()
    cap = 256
    while True:
        out = np.zeros(cap, N.TR_HIT_DTYPE)
        n = C.c_int32()
        rc = N.lib().cmgpu_tr_scan_hb(sc._model, semiring, C.byref(tt), C.byref(b), *[v.ctypes.data for v in vs],
                                      a.ctypes.data, a.size - 2, i0, j0, float(cutoff), int(bool(do_null3)),
                                      int(pass_idx), float(env_cutoff), C.byref(vsc), C.byref(vmode), C.byref(ei),
                                      C.byref(ej), out.ctypes.data, cap, C.byref(n))
        if rc == N.CMGPU_EOVERFLOW and n.value > cap:
            cap = n.value
            continue
        N.check(rc)
        return _tr_hits(out, n.value), vsc.value, vmode.value, ei.value, ej.value


def tr_cyk_scan_hb(cm, tri: TrInputs, bands: Bands, valid, dsq, i0: int, j0: int, cutoff: float, do_null3: bool,
                   pass_idx: int, env_cutoff: float):
    """src/cm_dpsearch_trunc.rs:264 -- (hits (i, j, score, bias, mode, root), vsc_root, vmode, envi, envj);
    valid = (jvalid, lvalid, rvalid, tvalid) per state."""
    sc = cm if isinstance(cm, Scanner) else _scanner(cm)
    return _tr_scan(sc, N.CYK_F32, tri, bands, valid, dsq, i0, j0, cutoff, do_null3, pass_idx, env_cutoff)


def ftr_inside_scan_hb(cm, tri: TrInputs, bands: Bands, valid, dsq, i0: int, j0: int, cutoff: float,
                       do_null3: bool, pass_idx: int, env_cutoff: float):
    """src/cm_dpsearch_trunc.rs:1055 -- the float Inside sibling of tr_cyk_scan_hb."""
    sc = cm if isinstance(cm, Scanner) else _scanner(cm)
    return _tr_scan(sc, N.INSIDE_F32, tri, bands, valid, dsq, i0, j0, cutoff, do_null3, pass_idx, env_cutoff)


_TR_RES_DTYPE = np.dtype({"names": ["vsc_root", "vmode", "envi", "envj", "hit_first", "nhits"],
                          "formats": [np.float32, np.int32, np.int64, np.int64, np.int64, np.int32],
                          "offsets": [0, 4, 8, 16, 24, 32], "itemsize": 40})


def tr_scan_hb_batch(sc: Scanner, semiring: int, tri: TrInputs, pass_idx: int, do_null3: bool, buf: np.ndarray,
                     tasks):
    """tasks: [(dsq_offset, i0, j0, env_cutoff, cutoff, Bands, (jvalid, lvalid, rvalid, tvalid))]
    -> [(hits, vsc, vmode, envi, envj)] per task."""
    b = np.ascontiguousarray(buf, np.uint8)
    tk = _task_array(tasks, 4)
    assert tk.dtype.itemsize == C.sizeof(N.TrTask)
    keep = []
    for q, t in enumerate(tasks):
        vs = [np.ascontiguousarray(x, np.uint8) for x in t[6]]
        keep.append(vs)
        tk["p"][q, 5:] = [v.ctypes.data for v in vs]
    tt = tri.struct()
    res = (N.TrResult * max(len(tasks), 1))()
    cap = 1024 + 16 * len(tasks)
    while True:
        out = np.zeros(cap, N.TR_HIT_DTYPE)
        n = C.c_int64()
        rc = N.lib().cmgpu_tr_scan_hb_batch(sc._model, None, semiring, C.byref(tt), int(pass_idx),
                                            int(bool(do_null3)), b.ctypes.data, b.size, tk.ctypes.data, len(tasks),
                                            res, out.ctypes.data, cap, C.byref(n))
        if rc == N.CMGPU_EOVERFLOW and n.value > cap:
            cap = n.value
            continue
        N.check(rc)
        r = _results(res, _TR_RES_DTYPE)[:len(tasks)]
        hl = out[:n.value].tolist()
        return [(hl[f:f + h], float(v), int(m), int(ei), int(ej)) for v, m, ei, ej, f, h in r.tolist()]


def _trq_scan(sc, semiring, qdbidx, tri: TrInputs, dsq, i0, j0, cutoff, do_null3, pass_idx):
    a = _frame(dsq)
    tt = tri.struct()
    vsc, vmode, bfull = C.c_float(), C.c_int32(), C.c_float()
    cap = 256
    while True:
        out = np.zeros(cap, N.TR_HIT_DTYPE)
        n = C.c_int32()
        rc = N.lib().cmgpu_tr_qdb_scan(sc._model, semiring, int(qdbidx), C.byref(tt), a.ctypes.data, a.size - 2, i0,
                                       j0, float(cutoff), int(bool(do_null3)), int(pass_idx), C.byref(vsc),
                                       C.byref(vmode), C.byref(bfull), out.ctypes.data, cap, C.byref(n))
        if rc == N.CMGPU_EOVERFLOW and n.value > cap:
            cap = n.value
            continue
        N.check(rc)
        return _tr_hits(out, n.value), vsc.value, vmode.value, bfull.value


def ref_tr_cyk_scan(cm, tri: TrInputs, dsq, i0: int, j0: int, cutoff: float, qdbidx: int, do_null3: bool,
                    pass_idx: int):
    """src/cm_dpsearch_trunc.rs:207 (generic_tr_scan, TrCYK) -- (hits (i, j, score, bias, mode, root),
    vsc_root, vmode, bsc_full); qdbidx N.NOQDB / N.QDB1 / N.QDB2."""
    sc = cm if isinstance(cm, Scanner) else _scanner(cm)
    return _trq_scan(sc, N.CYK_F32, qdbidx, tri, dsq, i0, j0, cutoff, do_null3, pass_idx)


def ref_itr_inside_scan(cm, tri: TrInputs, dsq, i0: int, j0: int, cutoff: float, qdbidx: int, do_null3: bool,
                        pass_idx: int):
    """src/cm_dpsearch_trunc.rs:226 (generic_tr_scan, integer TrInside) -- same results as ref_tr_cyk_scan;
    reads the integer tables tri.ilmesc / irmesc / ipty."""
    sc = cm if isinstance(cm, Scanner) else _scanner(cm)
    return _trq_scan(sc, N.INSIDE_I32, qdbidx, tri, dsq, i0, j0, cutoff, do_null3, pass_idx)


def tr_qdb_scan_batch(sc: Scanner, semiring: int, qdbidx: int, tri: TrInputs, pass_idx: int, do_null3: bool,
                      buf: np.ndarray, windows, cutoff: float):
    """Many windows in one call: windows is N.WINDOW_DTYPE (dsq_offset, i0, j0) into buf ->
    [(hits, vsc_root, vmode, bsc_full)] per window."""
    b = np.ascontiguousarray(buf, np.uint8)
    w = np.ascontiguousarray(windows, N.WINDOW_DTYPE)
    tt = tri.struct()
    res = (N.TrqResult * max(len(w), 1))()
    cap = 1024 + 16 * len(w)
    while True:
        out = np.zeros(cap, N.TR_HIT_DTYPE)
        n = C.c_int64()
        rc = N.lib().cmgpu_tr_qdb_scan_batch(sc._model, None, semiring, int(qdbidx), C.byref(tt), int(pass_idx),
                                             int(bool(do_null3)), b.ctypes.data, b.size, w.ctypes.data, len(w),
                                             float(cutoff), res, out.ctypes.data, cap, C.byref(n))
        if rc == N.CMGPU_EOVERFLOW and n.value > cap:
            cap = n.value
            continue
        N.check(rc)
        return [(_tr_hits(out[r.hit_first:], r.nhits), r.vsc_root, r.vmode, r.bsc_full) for r in res[:len(w)]]


def tr_qdb_stats(sc: Scanner):
    """(kernel ms, J-plane cells, launches) of the last truncated QDB call on this model."""
    ms, cells, launches = C.c_double(), C.c_int64(), C.c_int32()
    N.check(N.lib().cmgpu_tr_qdb_stats(sc._model, C.byref(ms), C.byref(cells), C.byref(launches)))
    return ms.value, cells.value, launches.value


# row of the truncated-begin penalties a pass uses (pty_idx_for_pass,
# src/cm_trunc.rs:99-107): 5'-and-3' (forced or any), 5'-only, 3'-only
PTY_ROW = {2: 1, 3: 2, 4: 0, 5: 0}


def truncated_tables(cm_s, local: bool) -> dict:
    """The truncated scanners' inputs of a CM (cmgpu_prep_truncated): marginal
    emissions lmesc/rmesc/ilmesc/irmesc [M*18], the penalty rows pty/ipty
    [3, M] of the local or global configuration, and lpos/rpos [M]."""
    from .model import params_struct
    M = cm_s.M
    out = dict(lmesc=np.zeros(M * 18, np.float32), rmesc=np.zeros(M * 18, np.float32),
               ilmesc=np.zeros(M * 18, np.int32), irmesc=np.zeros(M * 18, np.int32),
               pty=np.zeros((3, M), np.float32), ipty=np.zeros((3, M), np.int32),
               lpos=np.zeros(M, np.int32), rpos=np.zeros(M, np.int32))
    p, keep = params_struct(cm_s)
    t = N.TrPrep()
    for k in ("lmesc", "rmesc", "pty"):
        setattr(t, k, N.ptr(out[k], C.c_float))
    for k in ("ilmesc", "irmesc", "ipty", "lpos", "rpos"):
        setattr(t, k, N.ptr(out[k], C.c_int32))
    N.check(N.lib().cmgpu_prep_truncated(C.byref(p), int(bool(local)), C.byref(t)))
    del keep
    return out


def tr_inputs(cm_s, cfg, pass_idx: int, local: bool) -> TrInputs:
    """TrInputs of one truncated pass (PLI_PASS_*: 2 5'-only, 3 3'-only,
    4/5 5'-and-3') in the local or global configuration."""
    t = truncated_tables(cm_s, local)
    r = PTY_ROW[int(pass_idx)]
    return TrInputs(t["lmesc"], t["rmesc"], t["pty"][r].copy(), t["lpos"], t["rpos"], int(cfg.clen), bool(local),
                    t["ilmesc"], t["irmesc"], t["ipty"][r].copy())


def tr_qdb_set_deck_budget(sc: Scanner, nbytes: int) -> None:
    """Device memory the truncated QDB scan may hold in window decks at once
    (0: the default, 4 GiB)."""
    N.check(N.lib().cmgpu_tr_qdb_set_deck_budget(sc._model, int(nbytes)))
