"""F3 / F3b host parts, no GPU: the library's Forward profile and bias
tables equal the oracle's restatement of build_forward_filter /
build_bias_filter (src/cm_pipeline.rs:969-1120, :1683-1720) bit for bit on
the reference test's grid of random profiles; and the oracle's emulation of
the striped four-lane engine computes the Forward recurrence itself: it
agrees with a plain float64 recurrence in natural order to float rounding,
as the bias null does with a float64 two-state forward."""
import math

import numpy as np
import pytest

import oracle
from infernox_b200 import _native as N
from infernox_b200.p7 import FwdFilter, P7Profile, mean_composition

from p7_helpers import reference_grid


def test_tables_match_oracle_on_reference_grid():
    for p, _ in reference_grid(reps=2):
        compo = mean_composition(p)
        f = FwdFilter(p, compo, device=-1)
        rfv, tr, eo, t1 = f.tables()
        orfv, otr = oracle.fwd_tables(p.M, p.mat, p.trans)
        oeo, ot1 = oracle.bias_tables(compo, p.M)
        assert rfv.tobytes() == orfv.tobytes(), p.M
        assert tr.tobytes() == otr.tobytes(), p.M
        assert eo.tobytes() == oeo.tobytes() and t1.tobytes() == ot1.tobytes(), p.M
        # gap, nonresidue and missing codes emit nothing from a match state
        assert (rfv[1:, [4, 16, 17]] == 0).all()
        f.close()


def forward64(rfv, tr, dsq, L):
    """Local multihit Forward in odds space, natural order, float64."""
    M = len(rfv) - 1
    tbm, amm, aim, adm, tmi, tii, tmd, tdd = (tr[:, a].astype(np.float64) for a in range(8))
    pmove = 3.0 / (L + 3.0)
    ploop = 1.0 - pmove
    mp, ip, dp = np.zeros(M + 1), np.zeros(M + 1), np.zeros(M + 1)
    xn, xj, xb, xc, tot = 1.0, 0.0, pmove, 0.0, 0.0
    for i in range(1, L + 1):
        x = dsq[i]
        mc = np.zeros(M + 1)
        mc[1:] = (xb * tbm[1:] + mp[:-1] * amm[1:] + ip[:-1] * aim[1:] + dp[:-1] * adm[1:]) * rfv[1:, x]
        ic = mp * tmi + ip * tii
        dc = np.zeros(M + 1)
        for k in range(2, M + 1):
            dc[k] = mc[k - 1] * tmd[k - 1] + dc[k - 1] * tdd[k - 1]
        xe = mc[1:].sum() + dc[1:].sum()
        xn *= ploop
        xc = xc * ploop + xe * 0.5
        xj = xj * ploop + xe * 0.5
        xb = xj * pmove + xn * pmove
        if xe > 1e4:
            xn, xc, xj, xb = xn / xe, xc / xe, xj / xe, xb / xe
            mc, ic, dc = mc / xe, ic / xe, dc / xe
            tot += math.log(xe)
        mp, ip, dp = mc, ic, dc
    return tot + math.log(xc * pmove) if xc > 0 else -math.inf


def bias64(eo, t1, dsq, L):
    lf = float(L)
    p1 = lf / (lf + 1.0)
    t = np.array([[p1, 1 - p1], [t1[0], t1[1]]])
    f = np.array([0.999, 0.001]) * eo[dsq[1]]
    sc = 0.0
    for i in range(2, L + 1):
        s = f.sum()
        sc += math.log(s)
        f = (f / s) @ t * eo[dsq[i]]
    sc += math.log(f.sum())
    return sc + lf * math.log(p1) + math.log(1 - p1)


def test_oracle_striped_engine_is_the_forward_recurrence():
    worst = 0.0
    for p, seqs in reference_grid(reps=1)[::2]:
        rfv, tr = oracle.fwd_tables(p.M, p.mat, p.trans)
        compo = mean_composition(p)
        eo, t1 = oracle.bias_tables(compo, p.M)
        for d in seqs[:6]:
            L = len(d) - 2
            sc, _, _ = oracle.fwd_score_batch(p.M, p.mat, p.trans, d, [0], [L])
            ref = forward64(rfv, tr, d, L)
            if math.isinf(ref):
                assert math.isinf(sc[0]) and sc[0] < 0
                continue
            worst = max(worst, abs(float(sc[0]) - ref) / max(1.0, abs(ref)))
            bs, _ = oracle.bias_score_batch(compo, p.M, d, [0], [L])
            assert abs(float(bs[0]) - bias64(eo.astype(np.float64), t1, d, L)) < 1e-4 * max(1.0, L / 50)
    assert worst < 2e-6, worst


def test_build_rejects_empty_model():
    p = P7Profile(0, np.zeros((1, 4), np.float32), np.zeros((1, 7), np.float32))
    with pytest.raises(N.CmgpuError):
        FwdFilter(p, np.full(4, 0.25, np.float32), device=-1)


def test_oracle_cascade_merge_and_accounting():
    """The oracle's f3_filter_sequence: survivors merged into disjoint,
    non-abutting windows inside the chunk; with every gate open (P <= 1)
    the result is the merge of all F1 windows and every stage counts them
    all; tightening F3 only removes windows."""
    from p7_helpers import peaked_profile, planted_frame
    m = 80
    p, cons = peaked_profile(3, m, peak=0.6)
    fr = planted_frame(9, 20000, cons, 5)
    kw = dict(max_length=100, mmu=-9.0, mlambda=0.69)
    compo = mean_composition(p)
    open_w, open_a = oracle.f3_filter_sequence((m, p.mat, p.trans), compo, -6.0, 0.69, fr, 0.5, 1.0, 1.0, 96, **kw)
    f1w, _, _, _ = oracle.f1_msv_windows(m, p.mat, p.trans, 100, -9.0, 0.69, fr, [0], [20000], 0.5, 96)
    assert open_a["n_past_msv"] == len(f1w) == open_a["n_past_fwd"] == open_a["n_past_fwdbias"]
    assert open_a["pos_past_fwdbias"] == open_a["pos_past_msv"]
    merged = []
    for _, s, e in f1w:
        if merged and merged[-1][1] + 1 >= s:
            merged[-1][1] = e  # the reference takes the later window's end
        else:
            merged.append([s, e])
    assert [(s, e) for s, e, _ in open_w] == [tuple(x) for x in merged]
    tight_w, tight_a = oracle.f3_filter_sequence((m, p.mat, p.trans), compo, -6.0, 0.69, fr, 0.5, 0.01, 0.01, 96,
                                                 **kw)
    assert tight_a["n_past_fwdbias"] <= tight_a["n_past_fwd"] <= tight_a["n_past_msv"]
    assert 0 < len(tight_w) <= len(open_w)
    for (s, e, _), (s2, _, _) in zip(tight_w, tight_w[1:]):
        assert 1 <= s <= e <= 20000 and e + 1 < s2
    # every survivor lies inside a window of the open pass
    for s, e, _ in tight_w:
        assert any(a <= s and e <= b for a, b, _ in open_w)


def test_pipeline_thresholds_match_reference_test():
    """The reference's own thresholds_match_c_table cases (C's
    cm_pipeline_Create table), and the band edges of that table."""
    import json
    import os
    from infernox_b200.p7 import pipeline_thresholds
    kat = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "pipeline_kat.json")))
    assert len(kat["cases"]) == 3
    for c in kat["cases"]:
        t = pipeline_thresholds(c["z"])
        for k, v in c["want"].items():
            assert t[k] == v, (c["z"], k)
    assert pipeline_thresholds(1.999e6)["f3"] == 0.02 and pipeline_thresholds(2.0e6)["f3"] == 0.005
    assert pipeline_thresholds(20e9)["f1"] == 0.06 and pipeline_thresholds(19.9e9)["f1"] == 0.15


def test_oracle_sse_engine_equals_lane_by_lane():
    """The oracle's SSE2 engine (the timed CPU baseline, the reference's own
    x86 code path) gives the lane-by-lane emulation's bits: on the reference
    test's grid and on long windows with planted homologs around the M = 100
    switch of the D passes."""
    from p7_helpers import peaked_profile, planted_frame
    for p, seqs in reference_grid(reps=2):
        for d in seqs:
            L = len(d) - 2
            a = oracle.fwd_score_batch(p.M, p.mat, p.trans, d, [0], [L])
            b = oracle.fwd_score_batch(p.M, p.mat, p.trans, d, [0], [L], scalar=True)
            assert all(x.tobytes() == y.tobytes() for x, y in zip(a, b)), (p.M, L)
    for m in (29, 99, 100, 128, 257, 400, 1500):
        p, cons = peaked_profile(5 + m, m, peak=0.7)
        fr = planted_frame(m, 3000, cons, 3)
        a = oracle.fwd_score_batch(m, p.mat, p.trans, fr, [0], [3000])
        b = oracle.fwd_score_batch(m, p.mat, p.trans, fr, [0], [3000], scalar=True)
        assert all(x.tobytes() == y.tobytes() for x, y in zip(a, b)) and a[1][0] > 0


def test_abi_refuses_bad_arguments_before_any_device_work():
    """The Forward filter's entry points check their arguments first: null
    pointers, empty models, a stage without its filter, a host-only filter
    asked to score -- each an error code, no device touched."""
    import ctypes as C
    from p7_helpers import random_profile, Lcg
    L = N.lib()
    assert L.cmgpu_fwd_filter_build(None, None, 0.0, 1.0, -1, None) == N.CMGPU_EINVAL
    assert L.cmgpu_fwd_score_batch(None, None, None, 0, None, 0, None, None) == N.CMGPU_EINVAL
    p = random_profile(Lcg(3), 12)
    f = FwdFilter(p, np.full(4, 0.25, np.float32), device=-1)  # host tables only
    buf = np.full(12, 255, np.uint8)
    buf[1:11] = 1
    w = np.array([(0, 1, 10)], N.WINDOW_DTYPE)
    out = np.zeros(1, np.float32)
    assert L.cmgpu_fwd_score_batch(f._h, None, buf.ctypes.data, buf.size, w.ctypes.data, 1, out.ctypes.data,
                                   None) == N.CMGPU_EINVAL
    assert b"without a device" in L.cmgpu_last_error()
    cfg = N.F3Config()
    cfg.do_msv, cfg.cmw, cfg.do_fwd = 1, 30, 1
    n = C.c_int32()
    assert L.cmgpu_f3_filter(f._h, None, None, None, buf.ctypes.data, buf.size, w.ctypes.data, 1, C.byref(cfg),
                             None, 0, C.byref(n), None) == N.CMGPU_EINVAL
    assert b"without its filter" in L.cmgpu_last_error()
    assert L.cmgpu_fwd_filter_set_kernel(f._h, 7) == N.CMGPU_EINVAL
    f.close()
