"""TEST INFRASTRUCTURE ONLY: ctypes binding of the oracle (qdb_oracle.c,
hb_oracle.c, tr_oracle.c, trq_oracle.c, p7_oracle.c, msv_oracle.c,
prep_oracle.c, calib_oracle.c, fwd_oracle.c).

Used by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg as
the checker of the GPU scanner.  The product package never imports it.
Build with `make -C oracle` (or oracle.build()).
"""
from __future__ import annotations

import ctypes as C
import math
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")

HIT_DTYPE = np.dtype([("i", np.int32), ("j", np.int32), ("score", np.float32), ("bias", np.float32)])
ENV_DTYPE = np.dtype([("start", np.int32), ("end", np.int32)])

_lib = None


def build() -> str:
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def use_native() -> str:
    """Load the -march=native build (the timed CPU baseline) instead of the
    portable one; builds it on this machine.  Call before the first lib()."""
    global LIB_PATH
    if _lib is not None:
        raise RuntimeError("oracle.use_native() must come before the first oracle call")
    subprocess.run(["make", "-s", "-C", HERE, "native"], check=True)
    LIB_PATH = os.path.join(HERE, "_build_native", "liboracle.so")
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        srcs = [os.path.join(HERE, f) for f in ("qdb_oracle.c", "hb_oracle.c", "tr_oracle.c", "trq_oracle.c",
                                                "p7_oracle.c", "msv_oracle.c", "prep_oracle.c", "calib_oracle.c",
                                                "fwd_oracle.c")]
        if not os.path.exists(LIB_PATH) or any(os.path.getmtime(LIB_PATH) < os.path.getmtime(f) for f in srcs):
            native = os.path.basename(os.path.dirname(LIB_PATH)) == "_build_native"
            subprocess.run(["make", "-s", "-C", HERE] + (["native"] if native else []), check=True)
        L = C.CDLL(LIB_PATH)
        vp = C.c_void_p
        P = C.POINTER
        L.oracle_qdb_scan.argtypes = [vp, C.c_int, C.c_int, P(C.c_uint8), C.c_int32, C.c_int32,
                                      C.c_float, C.c_int, vp, C.c_int32, P(C.c_int32), vp, vp, vp,
                                      C.c_int32, P(C.c_int32), P(C.c_double), P(C.c_double)]
        L.oracle_cyk_seq_filter.argtypes = [vp, P(C.c_uint8), C.c_int32, C.c_float, C.c_int, vp,
                                            C.c_int32, P(C.c_int32)]
        L.oracle_final_stage_inside_opt.argtypes = [vp, P(C.c_uint8), vp, C.c_int32, C.c_float,
                                                    C.c_int, C.c_int, vp, C.c_int32, P(C.c_int32)]
        L.oracle_vit_score_batch.argtypes = [C.c_int, vp, vp, vp, vp, vp, C.c_int32, vp, vp]
        L.oracle_vit_score_batch_scalar.argtypes = [C.c_int, vp, vp, vp, vp, vp, C.c_int32, vp, vp]
        L.oracle_vit_tables.argtypes = [C.c_int, vp, vp, vp, vp]
        L.oracle_msv_tables.argtypes = [C.c_int, vp, vp, C.c_int, vp, vp, vp, vp, vp]
        L.oracle_msv_score_batch.argtypes = [C.c_int, vp, vp, C.c_int, vp, vp, vp, vp, C.c_int32, vp, vp]
        L.oracle_f1_msv_windows.argtypes = [C.c_int, vp, vp, C.c_int, C.c_double, C.c_double, vp, vp, vp,
                                            C.c_int32, C.c_double, C.c_int64, vp, vp, C.c_int64, vp, vp,
                                            C.c_int64, P(C.c_int64)]
        L.oracle_f1_msv_windows.restype = C.c_int64
        L.oracle_ssv_threshold.argtypes = [C.c_int, vp, vp, C.c_int, C.c_double, C.c_double, C.c_double]
        L.oracle_ssv_threshold.restype = C.c_int
        L.oracle_hb_scan.argtypes = [vp, C.c_int, vp, vp, vp, vp, vp, vp, C.c_int32, C.c_int32, C.c_float,
                                     C.c_int, C.c_float, C.c_int, P(C.c_float), P(C.c_int64), P(C.c_int64), vp,
                                     C.c_int32]
        L.oracle_tr_hb_scan.argtypes = [vp, C.c_int] + [vp] * 5 + [C.c_int32] + [vp] * 4 + [vp] * 5 + [
            vp, C.c_int32, C.c_int32, C.c_float, C.c_int, C.c_int, C.c_float, C.c_int, P(C.c_float), P(C.c_int32),
            P(C.c_int64), P(C.c_int64), vp, C.c_int32]
        L.oracle_trq_scan.argtypes = [vp, C.c_int] + [vp] * 8 + [C.c_int32, vp, C.c_int32, C.c_int32, C.c_float,
                                     C.c_int, C.c_int, C.c_int, C.c_int, P(C.c_float), P(C.c_int32),
                                     P(C.c_float), vp, C.c_int32]
        L.oracle_ilogsum_table.argtypes = [P(C.c_int32), C.c_int]
        L.oracle_ilogsum.argtypes = [C.c_int32, C.c_int32]
        L.oracle_ilogsum.restype = C.c_int32
        L.oracle_calib_scan.argtypes = [vp, C.c_int, C.c_int, P(C.c_uint8), C.c_int32, C.c_int32, C.c_int, vp,
                                        C.c_int32, P(C.c_int32), P(C.c_double)]
        L.oracle_genomic_sample.argtypes = [C.c_uint32, C.c_int32, C.c_int32, vp]
        L.oracle_exp_fit.argtypes = [vp, C.c_int64, C.c_int, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_float,
                                     C.c_double, vp]
        L.oracle_fwd_tables.argtypes = [C.c_int, vp, vp, vp, vp]
        L.oracle_fwd_score_batch.argtypes = [C.c_int, vp, vp, vp, vp, vp, C.c_int32, vp, vp, vp]
        L.oracle_fwd_score_batch_scalar.argtypes = [C.c_int, vp, vp, vp, vp, vp, C.c_int32, vp, vp, vp]
        L.oracle_bias_tables.argtypes = [vp, C.c_int, vp, vp]
        L.oracle_bias_score_batch.argtypes = [vp, C.c_int, vp, vp, vp, C.c_int32, vp, vp]
        _lib = L
    return _lib


def _u8(a):
    a = np.ascontiguousarray(a, np.uint8)
    return a, a.ctypes.data_as(C.POINTER(C.c_uint8))


def qdb_scan(cm, semiring, qdbidx, dsq, i0, j0, cutoff, do_null3, want_cands=False):
    """generic_scan restated: returns (hits, cands, cells, terms)."""
    L = lib()
    a, pa = _u8(dsq)
    cap = max(64, (j0 - i0 + 1) + 64)
    hits = np.zeros(cap, HIT_DTYPE)
    n = C.c_int32()
    cells, terms = C.c_double(), C.c_double()
    ccap = 0
    cj = cd = cs = None
    ncand = C.c_int32()
    if want_cands:
        ccap = max(1024, (j0 - i0 + 1) * (cm.W + 2))
        cj = np.zeros(ccap, np.int32)
        cd = np.zeros(ccap, np.int32)
        cs = np.zeros(ccap, np.float32)
    rc = L.oracle_qdb_scan(C.byref(cm.as_struct()), semiring, qdbidx, pa, i0, j0, float(cutoff),
                           int(bool(do_null3)), hits.ctypes.data, cap, C.byref(n),
                           cj.ctypes.data if want_cands else None,
                           cd.ctypes.data if want_cands else None,
                           cs.ctypes.data if want_cands else None, ccap,
                           C.byref(ncand) if want_cands else None, C.byref(cells), C.byref(terms))
    if rc != 0:
        raise RuntimeError(f"oracle overflow rc={rc}")
    out = [(int(h["i"]), int(h["j"]), float(h["score"]), float(h["bias"])) for h in hits[: n.value]]
    cands = None
    if want_cands:
        k = ncand.value
        cands = list(zip(cj[:k].tolist(), cd[:k].tolist(), cs[:k].tolist()))
    return out, cands, cells.value, terms.value


def cyk_seq_filter(cm, dsq, n, cutoff, do_null3):
    L = lib()
    a, pa = _u8(dsq)
    cap = 4096
    envs = np.zeros(cap, ENV_DTYPE)
    nout = C.c_int32()
    rc = L.oracle_cyk_seq_filter(C.byref(cm.as_struct()), pa, n, float(cutoff), int(bool(do_null3)),
                                 envs.ctypes.data, cap, C.byref(nout))
    if rc != 0:
        raise RuntimeError("oracle envelope overflow")
    return [(int(e["start"]), int(e["end"])) for e in envs[: nout.value]]


def final_stage_inside_opt(cm, dsq, envs, cutoff, do_null3, nonbanded):
    L = lib()
    a, pa = _u8(dsq)
    ev = np.asarray([tuple(e) for e in envs], ENV_DTYPE) if len(envs) else np.zeros(1, ENV_DTYPE)
    cap = 1 << 16
    hits = np.zeros(cap, HIT_DTYPE)
    nout = C.c_int32()
    rc = L.oracle_final_stage_inside_opt(C.byref(cm.as_struct()), pa, ev.ctypes.data, len(envs),
                                         float(cutoff), int(bool(do_null3)), int(bool(nonbanded)),
                                         hits.ctypes.data, cap, C.byref(nout))
    if rc != 0:
        raise RuntimeError("oracle hit overflow")
    return [(int(h["i"]), int(h["j"]), float(h["score"]), float(h["bias"])) for h in hits[: nout.value]]


def ilogsum_table(n=23000):
    t = np.zeros(n, np.int32)
    lib().oracle_ilogsum_table(t.ctypes.data_as(C.POINTER(C.c_int32)), n)
    return t


def ilogsum(a, b):
    return int(lib().oracle_ilogsum(a, b))


def vit_score_batch(M, mat, trans, buf, offs, lens, scalar=False):
    """vit_score on each sequence: (scores f32, scored u8; 0 = overflow);
    scalar: the scalar sweep (vit_score_scalar) instead of the SSE2 engine."""
    mat = np.ascontiguousarray(mat, np.float32)
    trans = np.ascontiguousarray(trans, np.float32)
    buf = np.ascontiguousarray(buf, np.uint8)
    offs = np.ascontiguousarray(offs, np.int64)
    lens = np.ascontiguousarray(lens, np.int32)
    sc = np.zeros(len(lens), np.float32)
    ok = np.zeros(len(lens), np.uint8)
    fn = lib().oracle_vit_score_batch_scalar if scalar else lib().oracle_vit_score_batch
    fn(int(M), mat.ctypes.data, trans.ctypes.data, buf.ctypes.data, offs.ctypes.data, lens.ctypes.data, len(lens),
       sc.ctypes.data, ok.ctypes.data)
    return sc, ok


def vit_tables(M, mat, trans):
    mat = np.ascontiguousarray(mat, np.float32)
    trans = np.ascontiguousarray(trans, np.float32)
    tab = np.zeros((M + 1) * 26, np.int16)
    sp = np.zeros(3, np.int16)
    lib().oracle_vit_tables(int(M), mat.ctypes.data, trans.ctypes.data, tab.ctypes.data, sp.ctypes.data)
    return tab, sp


def _f32(a):
    return np.ascontiguousarray(a, np.float32)


def msv_tables(M, mat, trans, max_length):
    """build_msv_filter restated: (rbv [(M+1)*18] u8, [base, bias, tbm, tec, tjb], prefix, suffix, scale_b)."""
    mat, trans = _f32(mat), _f32(trans)
    rbv = np.zeros((M + 1) * 18, np.uint8)
    b6 = np.zeros(6, np.uint8)
    pre = np.zeros(M + 1, np.float32)
    suf = np.zeros(M + 1, np.float32)
    sc = np.zeros(1, np.float32)
    lib().oracle_msv_tables(int(M), mat.ctypes.data, trans.ctypes.data, int(max_length), rbv.ctypes.data,
                            b6.ctypes.data, pre.ctypes.data, suf.ctypes.data, sc.ctypes.data)
    return rbv, b6[:5], pre, suf, sc[0]


def msv_score_batch(M, mat, trans, max_length, buf, offs, lens, wlen=None):
    """msv_score (wlen None) / msv_score_reconfig per frame: (scores f32, scored u8; 0 = overflow)."""
    mat, trans = _f32(mat), _f32(trans)
    buf = np.ascontiguousarray(buf, np.uint8)
    offs = np.ascontiguousarray(offs, np.int64)
    lens = np.ascontiguousarray(lens, np.int32)
    wl = None if wlen is None else np.ascontiguousarray(wlen, np.int32)
    sc = np.zeros(len(lens), np.float32)
    ok = np.zeros(len(lens), np.uint8)
    lib().oracle_msv_score_batch(int(M), mat.ctypes.data, trans.ctypes.data, int(max_length), buf.ctypes.data,
                                 offs.ctypes.data, lens.ctypes.data, None if wl is None else wl.ctypes.data,
                                 len(lens), sc.ctypes.data, ok.ctypes.data)
    return sc, ok


def f1_msv_windows(M, mat, trans, max_length, mmu, mlambda, buf, offs, lens, f1, cmw):
    """f1_msv_windows restated on each chunk: (windows [(chunk, start, end)], scores, raws [(chunk, n, length, k)],
    raw scores)."""
    mat, trans = _f32(mat), _f32(trans)
    buf = np.ascontiguousarray(buf, np.uint8)
    offs = np.ascontiguousarray(offs, np.int64)
    lens = np.ascontiguousarray(lens, np.int32)
    cap = 1024
    while True:
        out = np.zeros((cap, 3), np.int64)
        osc = np.zeros(cap, np.float32)
        raw = np.zeros((cap, 4), np.int64)
        rsc = np.zeros(cap, np.float32)
        nr = C.c_int64()
        n = lib().oracle_f1_msv_windows(int(M), mat.ctypes.data, trans.ctypes.data, int(max_length), float(mmu),
                                        float(mlambda), buf.ctypes.data, offs.ctypes.data, lens.ctypes.data,
                                        len(lens), float(f1), int(cmw), out.ctypes.data, osc.ctypes.data, cap,
                                        raw.ctypes.data, rsc.ctypes.data, cap, C.byref(nr))
        if n <= cap and nr.value <= cap:
            return out[:n], osc[:n], raw[: nr.value], rsc[: nr.value]
        cap = max(n, nr.value) + 16


def ssv_threshold(M, mat, trans, max_length, mmu, mlambda, f1):
    mat, trans = _f32(mat), _f32(trans)
    return int(lib().oracle_ssv_threshold(int(M), mat.ctypes.data, trans.ctypes.data, int(max_length), float(mmu),
                                          float(mlambda), float(f1)))


def fwd_tables(M, mat, trans):
    """build_forward_filter restated: (rfv [(M+1), 18], [(M+1), 8] = tbm, amm, aim, adm, tmi, tii, tmd, tdd)."""
    mat, trans = _f32(mat), _f32(trans)
    rfv = np.zeros((M + 1) * 18, np.float32)
    tr = np.zeros((M + 1) * 8, np.float32)
    lib().oracle_fwd_tables(int(M), mat.ctypes.data, trans.ctypes.data, rfv.ctypes.data, tr.ctypes.data)
    return rfv.reshape(M + 1, 18), tr.reshape(M + 1, 8)


def fwd_score_batch(M, mat, trans, buf, offs, lens, scalar=False):
    """forward_filter_score (striped engine) per frame: (scores, totscale, xc);
    scalar: the lane-by-lane emulation instead of the SSE2 one."""
    mat, trans = _f32(mat), _f32(trans)
    buf = np.ascontiguousarray(buf, np.uint8)
    offs = np.ascontiguousarray(offs, np.int64)
    lens = np.ascontiguousarray(lens, np.int32)
    n = len(lens)
    sc, ts, xc = (np.zeros(n, np.float32) for _ in range(3))
    fn = lib().oracle_fwd_score_batch_scalar if scalar else lib().oracle_fwd_score_batch
    fn(int(M), mat.ctypes.data, trans.ctypes.data, buf.ctypes.data, offs.ctypes.data, lens.ctypes.data, n,
       sc.ctypes.data, ts.ctypes.data, xc.ctypes.data)
    return sc, ts, xc


def bias_tables(compo, M):
    compo = _f32(compo)
    eo = np.zeros(36, np.float32)
    t1 = np.zeros(3, np.float32)
    lib().oracle_bias_tables(compo.ctypes.data, int(M), eo.ctypes.data, t1.ctypes.data)
    return eo.reshape(18, 2), t1


def bias_score_batch(compo, M, buf, offs, lens):
    """bias_filter_score per frame: (scores, the scores before the length term)."""
    compo = _f32(compo)
    buf = np.ascontiguousarray(buf, np.uint8)
    offs = np.ascontiguousarray(offs, np.int64)
    lens = np.ascontiguousarray(lens, np.int32)
    n = len(lens)
    sc, rows = np.zeros(n, np.float32), np.zeros(n, np.float32)
    lib().oracle_bias_score_batch(compo.ctypes.data, int(M), buf.ctypes.data, offs.ctypes.data, lens.ctypes.data, n,
                                  sc.ctypes.data, rows.ctypes.data)
    return sc, rows


def _null_one(L):
    """p7_bg_null_one (src/cm_pipeline.rs:1122-1125)."""
    p1 = L / (L + 1.0)
    return L * math.log(p1) + math.log(1.0 - p1)


def _exp_surv(x, mu, lam):
    """esl_exp_surv (src/cp9.rs:6531-6537)."""
    return 1.0 if x < mu else math.exp(-lam * (x - mu))


def _gumbel_surv(x, mu, lam):
    """esl_gumbel_surv (src/cm_pipeline.rs:1852-1861)."""
    y = lam * (x - mu)
    ey = -math.exp(-y)
    return -ey if abs(ey) < 5e-9 else 1.0 - math.exp(ey)


def f3_filter_sequence(p7, compo, ftau, flambda, chunk, f1, f3, f3b, cmw, msvbias=None, vit=None, do_fwd=True,
                       do_fwdbias=True, do_msv=True, maxw=0, max_length=0, mmu=0.0, mlambda=0.0):
    """f3_filter_sequence (src/cm_pipeline.rs:1863-2164) on one chunk (a frame
    [255, residues, 255]): the merged surviving windows [(start, end, score)]
    and the accounting dict.  p7 = (M, mat, trans); msvbias = (f1b, lmmu,
    lmlambda) or None; vit = (f2, do_vitbias, f2b, lvmu, lvlambda) or None."""
    M, mat, trans = p7
    chunk = np.ascontiguousarray(chunk, np.uint8)
    win_len = len(chunk) - 2
    ln2 = math.log(2.0)
    if do_msv:
        w, _, _, _ = f1_msv_windows(M, mat, trans, max_length, mmu, mlambda, chunk, [0], [win_len], f1, cmw)
        wins = [(int(s), int(e)) for _, s, e in w]
    else:
        n, mw = win_len, maxw
        nwin = 1
        if n > 2 * mw:
            nwin += (n - 2 * mw) // (mw + 1)
            if (n - 2 * mw) % (mw + 1) > 0:
                nwin += 1
        wins = [(1 + i * (mw + 1), min(1 + i * (mw + 1) + 2 * mw - 1, n)) for i in range(nwin)]
    nwin = len(wins)
    # one frame per window: [255, residues ws..we, 255]
    frames, offs, lens = [], [], []
    pos = 0
    for ws, we in wins:
        f = np.concatenate([[255], chunk[ws:we + 1], [255]]).astype(np.uint8)
        frames.append(f)
        offs.append(pos)
        lens.append(we - ws + 1)
        pos += len(f)
    buf = np.concatenate(frames) if frames else np.zeros(0, np.uint8)
    bias = bias_score_batch(compo, M, buf, offs, lens)[0] if nwin else np.zeros(0, np.float32)
    fwd = fwd_score_batch(M, mat, trans, buf, offs, lens)[0] if nwin and do_fwd else np.zeros(nwin, np.float32)
    msv = msv_score_batch(M, mat, trans, max_length, buf, offs, lens, lens) if nwin and msvbias else None
    vsc = vit_score_batch(M, mat, trans, buf, offs, lens) if nwin and vit else None
    s_f1b = [True] * nwin
    s_f2 = [True] * nwin
    s_f2b = [True] * nwin
    s_f3 = [False] * nwin
    s_f3b = [False] * nwin
    wb = [np.float32(-999.0)] * nwin
    for i in range(nwin):
        wlen = lens[i]
        nullsc = _null_one(wlen)
        if msvbias is not None and msv[1][i]:
            f1b, lmmu, lml = msvbias
            if _gumbel_surv((float(msv[0][i]) - float(bias[i])) / ln2, lmmu, lml) > f1b:
                s_f1b[i] = False
                continue
        if vit is not None and vsc[1][i]:
            f2, do_vitbias, f2b, lvmu, lvl = vit
            vf = float(vsc[0][i])
            if _gumbel_surv((vf - nullsc) / ln2, lvmu, lvl) > f2:
                s_f2[i] = s_f2b[i] = False
                continue
            if do_vitbias and _gumbel_surv((vf - float(bias[i])) / ln2, lvmu, lvl) > f2b:
                s_f2b[i] = False
                continue
        if do_fwd:
            wsc = (float(fwd[i]) - nullsc) / ln2
            wb[i] = np.float32(wsc)
            if _exp_surv(wsc, ftau, flambda) > f3:
                continue
        s_f3[i] = True
        if do_fwd and do_fwdbias:
            wsc = (float(fwd[i]) - float(bias[i])) / ln2
            wb[i] = np.float32(wsc)
            if _exp_surv(wsc, ftau, flambda) > f3b:
                continue
        s_f3b[i] = True
    ns = [wins[i][0] for i in range(nwin) if s_f3b[i]]
    ne = [wins[i][1] for i in range(nwin) if s_f3b[i]]
    nb = [wb[i] for i in range(nwin) if s_f3b[i]]
    out = []
    i = 0
    while i < len(ns):
        i2 = i + 1
        while i2 < len(ns) and ne[i] + 1 >= ns[i2]:
            ne[i] = ne[i2]
            nb[i] = max(nb[i], nb[i2])
            i2 += 1
        out.append((ns[i], ne[i], np.float32(nb[i])))
        i = i2
    acct = dict.fromkeys(("n_past_msv", "pos_past_msv", "n_past_msvbias", "pos_past_msvbias", "n_past_vit",
                          "pos_past_vit", "n_past_vitbias", "pos_past_vitbias", "n_past_fwd", "pos_past_fwd",
                          "n_past_fwdbias", "pos_past_fwdbias"), 0)
    acct["n_past_msv"] = nwin
    stages = (("msvbias", s_f1b), ("vit", s_f2), ("vitbias", s_f2b), ("fwd", s_f3), ("fwdbias", s_f3b))
    for i in range(nwin):
        wlen = lens[i]
        acct["pos_past_msv"] += wlen
        for name, s in stages:
            if s[i]:
                acct["n_past_" + name] += 1
                acct["pos_past_" + name] += wlen
        if i > 0:
            ov = wins[i - 1][1] - wins[i][0] + 1
            if ov > 0:
                acct["pos_past_msv"] -= ov
                for name, s in stages:
                    if s[i] and s[i - 1]:
                        acct["pos_past_" + name] -= ov
    return out, acct


def hb_scan(cm, inside, bands, dsq, i0, j0, env_cutoff, report, cutoff, do_null3):
    """fast_cyk_scan_hb_core / fast_finside_scan_hb restated: (vsc_root, envi, envj, hits).
    bands: (jmin, jmax, hd_off, hdmin, hdmax) int32 arrays."""
    a, _ = _u8(dsq)
    bs = [np.ascontiguousarray(x, np.int32) for x in bands]
    vsc, ei, ej = C.c_float(), C.c_int64(), C.c_int64()
    cap = 256
    while True:
        hits = np.zeros(cap, HIT_DTYPE)
        n = lib().oracle_hb_scan(C.byref(cm.as_struct()), int(bool(inside)), *[b.ctypes.data for b in bs],
                                 a.ctypes.data, i0, j0, float(env_cutoff), int(bool(report)), float(cutoff),
                                 int(bool(do_null3)), C.byref(vsc), C.byref(ei), C.byref(ej), hits.ctypes.data, cap)
        if n <= cap:
            out = [(int(h["i"]), int(h["j"]), float(h["score"]), float(h["bias"])) for h in hits[:n]]
            return vsc.value, ei.value, ej.value, out
        cap = n


TR_HIT_DTYPE = np.dtype([("i", np.int32), ("j", np.int32), ("score", np.float32), ("bias", np.float32),
                         ("mode", np.int32), ("root", np.int32)])


def tr_hb_scan(cm, inside, tt, valid, bands, dsq, i0, j0, cutoff, do_null3, pass_idx, env_cutoff, local):
    """tr_cyk_scan_hb / ftr_inside_scan_hb restated: (hits, vsc_root, vmode, envi, envj).
    tt: dict lmesc [M*18], rmesc, pty [M], lpos, rpos [M], clen; valid: (j, l, r, t) uint8 [M];
    bands: (jmin, jmax, hd_off, hdmin, hdmax)."""
    a, _ = _u8(dsq)
    f32 = lambda x: np.ascontiguousarray(x, np.float32)
    i32 = lambda x: np.ascontiguousarray(x, np.int32)
    lm, rm, pty = f32(tt["lmesc"]), f32(tt["rmesc"]), f32(tt["pty"])
    lp, rp = i32(tt["lpos"]), i32(tt["rpos"])
    vs = [np.ascontiguousarray(x, np.uint8) for x in valid]
    bs = [i32(x) for x in bands]
    vsc, vmode, ei, ej = C.c_float(), C.c_int32(), C.c_int64(), C.c_int64()
    cap = 256
    while True:
        hits = np.zeros(cap, TR_HIT_DTYPE)
        n = lib().oracle_tr_hb_scan(C.byref(cm.as_struct()), int(bool(inside)), lm.ctypes.data, rm.ctypes.data,
                                    pty.ctypes.data, lp.ctypes.data, rp.ctypes.data, int(tt["clen"]),
                                    *[v.ctypes.data for v in vs], *[b.ctypes.data for b in bs], a.ctypes.data,
                                    i0, j0, float(cutoff), int(bool(do_null3)), int(pass_idx), float(env_cutoff),
                                    int(bool(local)), C.byref(vsc), C.byref(vmode), C.byref(ei), C.byref(ej),
                                    hits.ctypes.data, cap)
        if n <= cap:
            out = [(int(h["i"]), int(h["j"]), float(h["score"]), float(h["bias"]), int(h["mode"]), int(h["root"]))
                   for h in hits[:n]]
            return out, vsc.value, vmode.value, ei.value, ej.value
        cap = n


def trq_scan(cm, inside, tt, dsq, i0, j0, cutoff, do_null3, qdbidx, pass_idx, local):
    """generic_tr_scan restated (ref_tr_cyk_scan / ref_itr_inside_scan): (hits, vsc_root, vmode, bsc_full).
    tt: dict with lmesc, rmesc, pty (float), ilmesc, irmesc, ipty (int), lpos, rpos, clen."""
    a, _ = _u8(dsq)
    f32 = lambda x: np.ascontiguousarray(x, np.float32)
    i32 = lambda x: np.ascontiguousarray(x, np.int32)
    arrs = [f32(tt["lmesc"]), f32(tt["rmesc"]), f32(tt["pty"]), i32(tt["ilmesc"]), i32(tt["irmesc"]),
            i32(tt["ipty"]), i32(tt["lpos"]), i32(tt["rpos"])]
    vsc, vmode, bfull = C.c_float(), C.c_int32(), C.c_float()
    cap = 256
    while True:
        hits = np.zeros(cap, TR_HIT_DTYPE)
        n = lib().oracle_trq_scan(C.byref(cm.as_struct()), int(bool(inside)), *[x.ctypes.data for x in arrs],
                                  int(tt["clen"]), a.ctypes.data, i0, j0, float(cutoff), int(bool(do_null3)),
                                  int(qdbidx), int(pass_idx), int(bool(local)), C.byref(vsc), C.byref(vmode),
                                  C.byref(bfull), hits.ctypes.data, cap)
        if n <= cap:
            out = [(int(h["i"]), int(h["j"]), float(h["score"]), float(h["bias"]), int(h["mode"]), int(h["root"]))
                   for h in hits[:n]]
            return out, vsc.value, vmode.value, bfull.value
        cap = n


# ---------------------------------------------------------------------------
# model preparation (prep_oracle.c)
# ---------------------------------------------------------------------------
def prep_configure(cm_s, local, W=0, beta1=1e-7, beta2=1e-15, betaW=1e-7):
    """The oracle's score tables and bands of a synthetic CM, as a dict of
    arrays with the fields of cmgpu_cm_scores (plus W, flags, el_selfsc,
    iel_selfsc)."""
    from infernox_b200 import _native as N
    from infernox_b200.model import params_struct
    M = cm_s.M
    out = dict(tsc=np.zeros((M, 6), np.float32), oesc=np.zeros((M, 324), np.float32),
               endsc=np.zeros(M, np.float32), beginsc=np.zeros(M, np.float32),
               itsc=np.zeros((M, 6), np.int32), ioesc=np.zeros((M, 324), np.int32),
               iendsc=np.zeros(M, np.int32), ibeginsc=np.zeros(M, np.int32),
               dmin1=np.zeros(M, np.int32), dmax1=np.zeros(M, np.int32),
               dmin2=np.zeros(M, np.int32), dmax2=np.zeros(M, np.int32),
               t_local=np.zeros((M, 6), np.float32))
    p, keep = params_struct(cm_s)
    s = N.CmScores()
    for k in ("tsc", "oesc", "endsc", "beginsc", "t_local"):
        setattr(s, k, N.ptr(out[k], C.c_float))
    for k in ("itsc", "ioesc", "iendsc", "ibeginsc", "dmin1", "dmax1", "dmin2", "dmax2"):
        setattr(s, k, N.ptr(out[k], C.c_int32))
    L = lib()
    L.oracle_prep_configure.argtypes = [C.c_void_p, C.c_int, C.c_int32, C.c_double, C.c_double, C.c_double,
                                        C.c_void_p]
    rc = L.oracle_prep_configure(C.byref(p), int(bool(local)), int(W), beta1, beta2, betaW, C.byref(s))
    if rc != 0:
        raise RuntimeError(f"oracle_prep_configure: {rc}")
    del keep
    out.update(W=int(s.W), flags=int(s.flags), el_selfsc=float(s.el_selfsc), iel_selfsc=int(s.iel_selfsc))
    return out


def prep_truncated(cm_s, local):
    """The oracle's truncated-scan inputs (the fields of cmgpu_tr_prep)."""
    from infernox_b200 import _native as N
    from infernox_b200.model import params_struct
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
    L = lib()
    L.oracle_prep_truncated.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
    rc = L.oracle_prep_truncated(C.byref(p), int(bool(local)), C.byref(t))
    if rc != 0:
        raise RuntimeError(f"oracle_prep_truncated: {rc}")
    del keep
    return out


def prep_cp9(cm_s):
    """The oracle's CP9 HMM of a CM (the fields of cmgpu_cp9)."""
    from infernox_b200 import _native as N
    from infernox_b200.model import params_struct
    H = cm_s.clen
    out = dict(mat=np.zeros((H + 1, 4), np.float32), ins=np.zeros((H + 1, 4), np.float32),
               t=np.zeros((H + 1, 10), np.float32), begin=np.zeros(H + 1, np.float32),
               end=np.zeros(H + 1, np.float32), msc=np.zeros((H + 1, 18), np.int32),
               isc=np.zeros((H + 1, 18), np.int32), otsc=np.zeros((H + 1, 12), np.int32),
               has_el=np.zeros(H + 1, np.uint8), hns2cs=np.zeros((H + 1, 3, 2), np.int32),
               el_pairs=np.zeros((cm_s.st.nodes, 2), np.int32))
    p, keep = params_struct(cm_s)
    s = N.Cp9()
    s.M = H
    for k, ct in (("mat", C.c_float), ("ins", C.c_float), ("t", C.c_float), ("begin", C.c_float),
                  ("end", C.c_float), ("msc", C.c_int32), ("isc", C.c_int32), ("otsc", C.c_int32),
                  ("has_el", C.c_uint8), ("hns2cs", C.c_int32), ("el_pairs", C.c_int32)):
        setattr(s, k, N.ptr(out[k], ct))
    L = lib()
    L.oracle_prep_cp9.argtypes = [C.c_void_p, C.c_void_p]
    rc = L.oracle_prep_cp9(C.byref(p), C.byref(s))
    if rc != 0:
        raise RuntimeError(f"oracle_prep_cp9: {rc}")
    del keep
    out["el_pairs"] = out["el_pairs"][: s.n_el]
    out["el_self"] = float(s.el_self)
    out["el_selfsc"] = int(s.el_selfsc)
    return out


# ---- cmcalibrate (calib_oracle.c, oracle_calib_scan in qdb_oracle.c) ------

EXP_DTYPE = np.dtype([("lambda", np.float64), ("mu", np.float64), ("dbsize", np.float64), ("mu_orig", np.float64),
                      ("tailp", np.float64), ("nrandhits", np.int32), ("pad", np.int32)])


def calib_scan(cm, semiring, qdbidx, dsq, i0, j0, do_null3, want_cells=False):
    """collect_scores's scan of one window: kept hits (i, j, score, bias)
    (and the DP cells computed, with want_cells)."""
    L = lib()
    a, pa = _u8(dsq)
    cap = max(64, (j0 - i0 + 1) + 64)
    hits = np.zeros(cap, HIT_DTYPE)
    n = C.c_int32()
    cells = C.c_double()
    rc = L.oracle_calib_scan(C.byref(cm.as_struct()), semiring, qdbidx, pa, i0, j0, int(bool(do_null3)),
                             hits.ctypes.data, cap, C.byref(n), C.byref(cells))
    if rc != 0:
        raise RuntimeError(f"oracle overflow rc={rc}")
    out = [(int(h["i"]), int(h["j"]), float(h["score"]), float(h["bias"])) for h in hits[: n.value]]
    return (out, cells.value) if want_cells else out


def genomic_sample(seed, L, nseq):
    """nseq frames [255, L residues, 255] of the genomic HMM, back to back."""
    out = np.zeros(nseq * (L + 2), np.uint8)
    lib().oracle_genomic_sample(seed, L, nseq, out.ctypes.data)
    return out


def exp_fit(scores, exp_mode, n_seqs, L, gtailn=250, ltailn=750, tailp=0.0, dbsize=0.0):
    """fit_histogram + set_exp_info; None where the reference errors."""
    s = np.ascontiguousarray(scores, np.float32)
    out = np.zeros(1, EXP_DTYPE)
    rc = lib().oracle_exp_fit(s.ctypes.data, len(s), exp_mode, n_seqs, L, gtailn, ltailn, float(tailp),
                              float(dbsize), out.ctypes.data)
    return None if rc else out[0]
