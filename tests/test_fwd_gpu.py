"""GPU F3 Forward and F3b composition-bias filters vs the oracle's
restatement of the reference's default striped engine and two-state null
(src/cm_pipeline.rs:1270-1418, :1722-1790): f32 score bits equal on the
reference test's grid of random profiles and sequences (every M around the
vector boundaries, L from 1 to 500, residue codes 0..15), on long windows
of large models with planted homologs (many rescalings), and the whole
f3_filter_sequence cascade (F1 SSV windows or tiles, F1b, F2 / F2b, F3 /
F3b gates, merge, residue accounting) window for window."""
import numpy as np
import pytest

import oracle
from infernox_b200 import _native as N
from infernox_b200.p7 import (FwdFilter, MsvFilter, VitFilter, bias_filter_score, f3_filter_batch,
                              f3_filter_sequence, forward_filter_score, mean_composition)

from p7_helpers import LS, Lcg, peaked_profile, planted_frame, random_profile, reference_grid

pytestmark = pytest.mark.gpu


def frames_of(seqs):
    bufs, wins, offs, lens, off = [], [], [], [], 0
    for d in seqs:
        l = len(d) - 2
        f = d.copy()
        f[0] = f[-1] = 255
        bufs.append(f)
        wins.append((off, 1, l))
        offs.append(off)
        lens.append(l)
        off += len(f)
    return np.concatenate(bufs), np.array(wins, N.WINDOW_DTYPE), offs, lens


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


@pytest.mark.parametrize("shared", [False, True], ids=["auto", "shared"])
def test_fwd_and_bias_match_oracle_on_reference_grid(shared):
    n = 0
    for p, seqs in reference_grid():
        buf, wins, offs, lens = frames_of(seqs)
        compo = mean_composition(p)
        f = FwdFilter(p, compo)
        f.set_kernel(shared)
        fs, bs = f.score_batch(buf, wins)
        ofs, _, _ = oracle.fwd_score_batch(p.M, p.mat, p.trans, buf, offs, lens)
        obs, _ = oracle.bias_score_batch(compo, p.M, buf, offs, lens)
        assert np.array_equal(bits(fs), bits(ofs)), (p.M, fs, ofs)
        assert np.array_equal(bits(bs), bits(obs)), (p.M, bs, obs)
        f.close()
        n += len(seqs)
    assert n == 21 * 8 * len(LS)


@pytest.mark.parametrize("shared", [False, True], ids=["auto", "shared"])
@pytest.mark.parametrize("m", [29, 99, 100, 120, 128, 256, 400, 1500])
def test_fwd_long_windows_planted_homologs(m, shared):
    """Long windows with planted consensus runs: the Forward mass grows past
    the 1e4 rescaling threshold many times; M = 99 / 100 straddle the switch
    from four fixed D passes to the early-stopping ones."""
    p, cons = peaked_profile(7 + m, m, peak=0.7)
    seqs = [planted_frame(31 + m + q, l, cons, n) for q, (l, n) in enumerate([(1, 0), (300, 1), (2500, 4),
                                                                            (20000, 12)])]
    buf, wins, offs, lens = frames_of(seqs)
    compo = mean_composition(p)
    f = FwdFilter(p, compo)
    f.set_kernel(shared)
    fs, bs = f.score_batch(buf, wins)
    ofs, ots, _ = oracle.fwd_score_batch(m, p.mat, p.trans, buf, offs, lens)
    obs, _ = oracle.bias_score_batch(compo, m, buf, offs, lens)
    assert np.array_equal(bits(fs), bits(ofs)), (fs, ofs)
    assert np.array_equal(bits(bs), bits(obs)), (bs, obs)
    assert ots[-1] > 0  # the longest window was rescaled
    ms, cells, launches = f.stats()
    assert cells == sum(lens) * m and launches == 2
    # single-window mirrors
    one = buf[wins[2]["dsq_offset"]:]
    assert np.float32(forward_filter_score(f, one, int(wins[2]["j0"]))).tobytes() == ofs[2].tobytes()
    assert np.float32(bias_filter_score(f, one, int(wins[2]["j0"]))).tobytes() == obs[2].tobytes()
    f.close()


def test_fwd_windows_inside_frames_in_any_order():
    """Windows cut from one frame at any offsets, uneven lengths, one empty."""
    rng = Lcg(77)
    p = random_profile(rng, 64)
    r = np.random.default_rng(3)
    fr = np.full(6002, 255, np.uint8)
    fr[1:-1] = r.integers(0, 16, 6000)
    cuts = [(1, 6000), (17, 400), (3000, 2999), (5999, 6000), (250, 4000), (1, 1)]
    wins = np.array([(0, a, b) for a, b in cuts], N.WINDOW_DTYPE)
    compo = np.array([0.4, 0.1, 0.1, 0.4], np.float32)
    f = FwdFilter(p, compo)
    fs, bs = f.score_batch(fr, wins)
    offs = [a - 1 for a, _ in cuts]
    lens = [max(0, b - a + 1) for a, b in cuts]
    ofs, _, _ = oracle.fwd_score_batch(64, p.mat, p.trans, fr, offs, lens)
    obs, _ = oracle.bias_score_batch(compo, 64, fr, offs, lens)
    assert np.array_equal(bits(fs), bits(ofs))
    assert np.array_equal(bits(bs), bits(obs))
    assert np.isneginf(fs[2]) and bs[2] == 0.0  # the empty window, as the reference scores it


F3_CASES = [
    # m, f1, f3, f3b, length, chunks, plants, stages
    (120, 0.35, 0.02, 0.02, 30000, 3, 6, "default"),
    (64, 0.5, 0.2, 0.1, 20000, 2, 8, "vit"),
    (90, 0.5, 0.3, 0.3, 12000, 2, 4, "msvbias"),
    (120, 0.35, 0.05, 0.05, 15000, 2, 5, "tiles"),
    (200, 0.4, 1.0, 1.0, 10000, 1, 3, "nofwd"),
]


@pytest.mark.parametrize("case", F3_CASES, ids=[c[-1] for c in F3_CASES])
def test_f3_filter_matches_oracle(case):
    m, f1, f3, f3b, l, nch, nplant, stages = case
    p, cons = peaked_profile(41 + m, m, peak=0.6)
    seqs = [planted_frame(500 + q, l, cons, nplant) for q in range(nch)]
    buf, wins, offs, lens = frames_of(seqs)
    compo = mean_composition(p)
    maxl, cmw = int(1.25 * m), max(1, int(1.2 * m))
    mmu, mlam, ftau, flam = -9.0, 0.69, -6.0, 0.69
    mf = MsvFilter(p, maxl, mmu, mlam)
    ff = FwdFilter(p, compo, ftau, flam)
    vf = VitFilter(p) if stages == "vit" else None
    kw = {}
    okw = {}
    if stages == "vit":
        kw["vit"] = okw["vit"] = (0.3, True, 0.3, -8.5, 0.69)
        kw["vf"] = vf
    if stages == "msvbias":
        kw["msvbias"] = okw["msvbias"] = (0.3, mmu, mlam)
    if stages == "tiles":
        kw["do_msv"] = okw["do_msv"] = False
        kw["maxw"] = okw["maxw"] = 2 * m
    if stages == "nofwd":
        kw["do_fwd"] = okw["do_fwd"] = False
    got, acct = f3_filter_batch(ff, buf, wins, f1, f3, f3b, cmw, mf=mf, **kw)
    want, wacct = [], {}
    for c, (o, n) in enumerate(zip(offs, lens)):
        ws, a = oracle.f3_filter_sequence((m, p.mat, p.trans), compo, ftau, flam, buf[o:o + n + 2], f1, f3, f3b, cmw,
                                          max_length=maxl, mmu=mmu, mlambda=mlam, **okw)
        want += [(c, s, e, sc) for s, e, sc in ws]
        for k, v in a.items():
            wacct[k] = wacct.get(k, 0) + v
    assert [(int(r["chunk"]), int(r["start"]), int(r["end"])) for r in got] == [w[:3] for w in want]
    assert np.array_equal(bits(got["score"]), bits([w[3] for w in want]))
    assert acct == wacct
    assert acct["n_past_msv"] > 0 and acct["n_past_fwdbias"] <= acct["n_past_fwd"] <= acct["n_past_msv"]
    if stages == "default":
        assert 0 < len(got) and acct["n_past_fwd"] < acct["n_past_msv"]
        one, oacct = f3_filter_sequence(mf, ff, buf[offs[0]:offs[0] + lens[0] + 2], lens[0], f1, f3, f3b, cmw)
        assert [(s, e) for s, e, _ in one] == [(w[1], w[2]) for w in want if w[0] == 0]
    for x in (mf, ff, vf):
        if x is not None:
            x.close()


def test_fwd_rejects_bad_windows():
    rng = Lcg(5)
    p = random_profile(rng, 20)
    f = FwdFilter(p, np.full(4, 0.25, np.float32))
    buf = np.full(12, 255, np.uint8)
    buf[1:11] = 2
    with pytest.raises(N.CmgpuError):
        f.score_batch(buf, np.array([(0, 1, 11)], N.WINDOW_DTYPE))  # past the buffer
    bad = buf.copy()
    bad[4] = 19
    with pytest.raises(N.CmgpuError):
        f.score_batch(bad, np.array([(0, 1, 10)], N.WINDOW_DTYPE))
    with pytest.raises(N.CmgpuError):
        f3_filter_batch(f, buf, np.array([(0, 1, 10)], N.WINDOW_DTYPE), 0.3, 0.1, 0.1, 30)  # SSV on, no MSV filter
    f.close()
