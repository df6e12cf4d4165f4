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
