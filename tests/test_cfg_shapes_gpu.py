"""The scanners at the model shapes of the benchmark workloads, against the
oracle, through the C ABI.

* cfg0 -- the --nohmm CYK workload: 72 columns, a 7 bp closing stem around
  three 5 bp hairpins; QDB1 CYK filter then QDB2 Inside on its envelopes,
  local configuration, both strands of a sequence with planted homologs.
* cfg3 -- the bifurcation-heavy truncated workload: 1500 columns, 60% of
  them paired, 25 bifurcations (M = 4629 states, W = 1551 for this seeded
  model).  Every scanner family on short windows (the oracle's full decks
  bound the sizes the tests can afford): the QDB1 CYK and non-banded integer
  Inside scans cell by cell, the HMM-banded CYK / float Inside scans, the
  truncated HMM-banded TrCYK / TrInside scans and the truncated QDB /
  non-banded TrCYK / TrInside scans.

Exact equality of every score's bits, as in the other parity tests.
"""
import numpy as np
import pytest

import oracle
from infernox_b200 import _native as N
from infernox_b200 import synth
from infernox_b200.hb import (TrInputs, fast_fcyk_scan_hb, fast_finside_scan_hb, ftr_inside_scan_hb,
                              ref_itr_inside_scan, ref_tr_cyk_scan, tr_cyk_scan_hb)
from infernox_b200.scan import CYK_F32, INSIDE_I32, KERNEL_SWEEP, NOQDB, QDB1, QDB2, Scanner

from hb_helpers import as_tuple, tr_tables, tr_valid, truncated_window, wide_bands
from helpers import frame, models, planted_seq

pytestmark = pytest.mark.gpu


def bits(x):
    return np.float32(x).tobytes()


def hit_bits(h):
    return [(x[0], x[1], bits(x[2]), bits(x[3])) for x in h]


def test_cfg0_nohmm_pipeline_both_strands():
    cm, g, l = models("cfg0")
    seq = planted_seq(cm, 20000, 0.5, 6, seed=2001)
    sc = Scanner(l)
    for strand in (seq, synth.revcomp(seq)):
        dsq = frame(strand)
        n = len(strand)
        env_ref = oracle.cyk_seq_filter(l, dsq, n, 0.0, True)
        env = sc.cyk_seq_filter(dsq, n, 0.0, True)
        assert env == env_ref and len(env) > 0
        ref = oracle.final_stage_inside_opt(l, dsq, env, 0.0, True, False)
        got = sc.final_stage_inside_opt(dsq, env, 0.0, True, False)
        assert [(h.i, h.j, bits(h.score), bits(h.bias)) for h in got] == hit_bits(ref) and ref
    sc.close()


def _cells(sc, cfg, sr, band, dsq, n):
    _, ref, _, _ = oracle.qdb_scan(cfg, sr, band, dsq, 1, n, -1e30, False, want_cands=True)
    got = sc.scan_cells(sr, band, dsq, 1, n, -1e30)
    rmap = {(j, d): s for j, d, s in ref}
    gmap = {(j, d): s for j, d, s in got}
    bad = [k for k in sorted(set(rmap) | set(gmap))
           if bits(gmap.get(k, np.nan)) != bits(rmap.get(k, np.nan))]
    return len(ref), bad


@pytest.mark.parametrize("sr,band,n", [(CYK_F32, QDB1, 300), (INSIDE_I32, QDB2, 200), (INSIDE_I32, NOQDB, 90)])
def test_cfg3_qdb_scan_every_cell(sr, band, n):
    cm, g, l = models("cfg3")
    assert l.M > 4000 and l.W > 1500
    dsq = frame(planted_seq(cm, n, 0.55, 0, seed=2003))
    sc = Scanner(l)
    nref, bad = _cells(sc, l, sr, band, dsq, n)
    assert nref > 0 and not bad, bad[:8]
    sc.close()


def test_cfg3_qdb_scan_hits_and_sweep_scope():
    """QDB1 CYK hits on a window holding the 3' part of a homolog; the node
    sweep kernel declines W > 255 with a clear error."""
    cm, g, l = models("cfg3")
    rng = np.random.default_rng(2005)
    h = synth.emit(cm, rng)
    seq = np.concatenate([synth.random_dsq(150, 0.55, rng), h[-250:], synth.random_dsq(100, 0.55, rng)])
    dsq = frame(seq)
    n = len(seq)
    sc = Scanner(l)
    ref, _, _, _ = oracle.qdb_scan(l, CYK_F32, QDB1, dsq, 1, n, -20.0, True)
    got = sc.generic_scan(CYK_F32, QDB1, dsq, 1, n, -20.0, True)
    assert [(x.i, x.j, bits(x.score), bits(x.bias)) for x in got] == hit_bits(ref) and ref
    sc.set_kernel(KERNEL_SWEEP)
    with pytest.raises(N.CmgpuError, match="W above"):
        sc.generic_scan(CYK_F32, QDB1, dsq, 1, n, -20.0, True)
    sc.close()


def test_cfg3_hb_scans():
    cm, g, l = models("cfg3")
    seq = frame(planted_seq(cm, 200, 0.55, 0, seed=2007))
    sc = Scanner(l)
    i0, j0 = 61, 130
    b = wide_bands(l, i0, j0)
    for cutoff, null3 in ((-20.0, True), (0.0, False)):
        ro = oracle.hb_scan(l, False, as_tuple(b), seq, i0, j0, -10.0, True, cutoff, null3)
        rg = fast_fcyk_scan_hb(sc, b, seq, i0, j0, -10.0, cutoff, null3)
        assert (bits(rg[0]), rg[1], rg[2]) == (bits(ro[0]), ro[1], ro[2])
        assert hit_bits(rg[3]) == hit_bits(ro[3])
        ro = oracle.hb_scan(l, True, as_tuple(b), seq, i0, j0, -10.0, True, cutoff, null3)
        rg = fast_finside_scan_hb(sc, b, seq, i0, j0, -10.0, cutoff, null3)
        assert (bits(rg[0]), rg[1], rg[2]) == (bits(ro[0]), ro[1], ro[2])
        assert hit_bits(rg[3]) == hit_bits(ro[3])
    sc.close()


@pytest.mark.parametrize("pass_idx", [2, 4])
def test_cfg3_truncated_scans(pass_idx):
    cm, g, l = models("cfg3")
    loc = True
    tt = tr_tables(cm, l, pass_idx, loc)
    tri = TrInputs(tt["lmesc"], tt["rmesc"], tt["pty"], tt["lpos"], tt["rpos"], tt["clen"], loc,
                   tt["ilmesc"], tt["irmesc"], tt["ipty"])
    sc = Scanner(l)
    f, i0, j0 = truncated_window(cm, l, pass_idx, 2009 + pass_idx, max_len=70)
    # truncated HMM-banded scans over wide bands
    b = wide_bands(l, i0, j0)
    valid = tr_valid(l.M, 5, pass_idx, True)
    for inside, fn in ((False, tr_cyk_scan_hb), (True, ftr_inside_scan_hb)):
        ro = oracle.tr_hb_scan(l, inside, tt, valid, as_tuple(b), f, i0, j0, -10.0, True, pass_idx, -5.0, loc)
        rg = fn(sc, tri, b, valid, f, i0, j0, -10.0, True, pass_idx, -5.0)
        assert (bits(rg[1]), rg[2], rg[3], rg[4]) == (bits(ro[1]), ro[2], ro[3], ro[4]), inside
        assert [(i, j, bits(s), bits(x), m, r) for i, j, s, x, m, r in rg[0]] == \
               [(i, j, bits(s), bits(x), m, r) for i, j, s, x, m, r in ro[0]], inside
    # truncated QDB / non-banded scans
    for qdb in (QDB1, NOQDB):
        for inside, fn in ((False, ref_tr_cyk_scan), (True, ref_itr_inside_scan)):
            ro = oracle.trq_scan(l, inside, tt, f, i0, j0, -10.0, True, qdb, pass_idx, loc)
            go = fn(sc, tri, f, i0, j0, -10.0, qdb, True, pass_idx)
            assert bits(go[1]) == bits(ro[1]) and go[2] == ro[2], (qdb, inside)
            assert bits(go[3]) == bits(ro[3]), (qdb, inside)
            assert [(i, j, bits(s), bits(x), m, r) for i, j, s, x, m, r in go[0]] == \
                   [(i, j, bits(s), bits(x), m, r) for i, j, s, x, m, r in ro[0]], (qdb, inside)
    sc.close()
