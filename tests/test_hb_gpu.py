"""GPU HMM-banded scanners vs the oracle (fast_cyk_scan_hb_core and
fast_finside_scan_hb restated), through the C ABI.

Equal bits of vsc_root, equal envelope bounds, and equal reported hits
(i, j, score bits, bias bits) for CYK (filter and hit-reporting forms) and
float Inside, global and local configurations, five model shapes, on wide
bands (the reference's own fixture), QDB-shaped bands, ragged bands and
nested (i, j) rectangles turned into d-bands as ij2d_bands builds them;
then many envelopes with their own bands in one batched call.
"""
import numpy as np
import pytest

import oracle
from infernox_b200 import _native as N
from infernox_b200.hb import fast_cyk_scan_hb, fast_fcyk_scan_hb, fast_finside_scan_hb, hb_scan_batch, hb_stats
from infernox_b200.scan import Scanner

from hb_helpers import as_tuple, qdb_bands, ragged_bands, rect_bands, wide_bands
from helpers import frame, models, planted_seq

pytestmark = pytest.mark.gpu

BANDS = {
    "wide": lambda cm, i0, j0, s: wide_bands(cm, i0, j0),
    "qdb": lambda cm, i0, j0, s: qdb_bands(cm, i0, j0),
    "ragged": lambda cm, i0, j0, s: ragged_bands(cm, i0, j0, s),
    "rect": lambda cm, i0, j0, s: rect_bands(cm, i0, j0, s),
}

CASES = [(m, loc, kind) for m in ("trna", "small0", "small2", "mb3") for loc in (False, True)
         for kind in ("wide", "qdb", "ragged", "rect")] + [("cfg2", True, "qdb"), ("cfg2", False, "ragged")]


def bits(x):
    return np.float32(x).tobytes()


def hits_bits(h):
    return [(i, j, bits(s), bits(b)) for i, j, s, b in h]


@pytest.mark.parametrize("case", CASES, ids=[f"{m}-{'loc' if l else 'glob'}-{k}" for m, l, k in CASES])
def test_hb_scans_match_oracle(case):
    name, loc, kind = case
    cm, g, l = models(name)
    cfg = l if loc else g
    seed = 31 + CASES.index(case)
    seq = frame(planted_seq(cm, 600, 0.5, 3, seed=seed, degenerate=0.01))
    sc = Scanner(cfg)
    w = min(cfg.W, 150)
    for i0 in (1, 200, 600 - w + 1):
        j0 = i0 + w - 1
        b = BANDS[kind](cfg, i0, j0, seed + i0)
        for env_cut in (-1e30, 0.0):
            vo, eio, ejo, _ = oracle.hb_scan(cfg, False, as_tuple(b), seq, i0, j0, env_cut, False, 0.0, False)
            vg, eig, ejg = fast_cyk_scan_hb(sc, b, seq, i0, j0, env_cut)
            assert (bits(vg), eig, ejg) == (bits(vo), eio, ejo), (i0, env_cut)
        for cutoff, null3 in ((-5.0, True), (0.0, False)):
            ro = oracle.hb_scan(cfg, False, as_tuple(b), seq, i0, j0, 0.0, True, cutoff, null3)
            rg = fast_fcyk_scan_hb(sc, b, seq, i0, j0, 0.0, cutoff, null3)
            assert (bits(rg[0]), rg[1], rg[2]) == (bits(ro[0]), ro[1], ro[2])
            assert hits_bits(rg[3]) == hits_bits(ro[3]), (i0, cutoff)
            ro = oracle.hb_scan(cfg, True, as_tuple(b), seq, i0, j0, 0.0, True, cutoff, null3)
            rg = fast_finside_scan_hb(sc, b, seq, i0, j0, 0.0, cutoff, null3)
            assert (bits(rg[0]), rg[1], rg[2]) == (bits(ro[0]), ro[1], ro[2])
            assert hits_bits(rg[3]) == hits_bits(ro[3]), (i0, cutoff)
    sc.close()


@pytest.mark.parametrize("semiring", [N.CYK_F32, N.INSIDE_F32])
def test_hb_batch_many_envelopes(semiring):
    cm, g, l = models("trna")
    rng = np.random.default_rng(5)
    frames, tasks, ref, off = [], [], [], 0
    sc = Scanner(l)
    kinds = list(BANDS)
    for q in range(24):
        n = int(rng.integers(80, 400))
        f = frame(planted_seq(cm, n, 0.5, 1, seed=500 + q))
        w = int(rng.integers(20, min(n, l.W) + 1))
        i0 = int(rng.integers(1, n - w + 2))
        j0 = i0 + w - 1
        b = BANDS[kinds[q % 4]](l, i0, j0, q)
        tasks.append((off, i0, j0, -2.0, -3.0, b))
        ref.append(oracle.hb_scan(l, semiring == N.INSIDE_F32, as_tuple(b), f, i0, j0, -2.0, True, -3.0, True))
        frames.append(f)
        off += len(f)
    buf = np.concatenate(frames)
    got = hb_scan_batch(sc, semiring, True, True, buf, tasks)
    nh = 0
    for (vg, eig, ejg, hg), (vo, eio, ejo, ho) in zip(got, ref):
        assert (bits(vg), eig, ejg) == (bits(vo), eio, ejo)
        assert hits_bits(hg) == hits_bits(ho)
        nh += len(ho)
    assert nh > 0
    ms, cells, launches = hb_stats(sc)
    assert cells > 0 and launches >= 1
    sc.close()


def test_hb_rejects_bad_bands():
    cm, g, l = models("small0")
    sc = Scanner(l)
    seq = frame(planted_seq(cm, 100, 0.5, 0, seed=1))
    b = wide_bands(l, 1, 60)
    bad = wide_bands(l, 1, 60)
    bad.hdmax = bad.hdmax.copy()
    bad.hdmax[bad.hd_off[1] + 5] = 30  # i = j - d + 1 < i0
    with pytest.raises(N.CmgpuError):
        fast_cyk_scan_hb(sc, bad, seq, 1, 60, 0.0)
    with pytest.raises(N.CmgpuError):
        fast_cyk_scan_hb(sc, b, seq, 1, 200, 0.0)  # beyond the sequence
    sc.close()
