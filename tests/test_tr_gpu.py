"""GPU truncated HMM-banded scanners vs the oracle (tr_cyk_scan_hb and
ftr_inside_scan_hb restated), through the C ABI.

Equal bits of vsc_root with its marginal mode, equal envelope bounds and
equal reported hits (i, j, score bits, bias bits, mode, entry state) after
overlap removal, for TrCYK and float TrInside, in the truncated passes
5'-only, 3'-only and 5'-and-3' (forced and any), global and local
truncation rules, on windows that cut a sampled homolog at the 5' end, the
3' end or both, with wide, ragged and QDB-shaped bands and dense or sparse
J/L/R/T plane validity; then a batch of envelopes in one call.
"""
import numpy as np
import pytest

import oracle
from infernox_b200 import _native as N
from infernox_b200 import synth
from infernox_b200.hb import TrInputs, ftr_inside_scan_hb, tr_cyk_scan_hb, tr_scan_hb_batch
from infernox_b200.scan import Scanner

from hb_helpers import as_tuple, qdb_bands, ragged_bands, tr_tables, tr_valid, truncated_window, wide_bands
from helpers import frame, models

pytestmark = pytest.mark.gpu

BANDS = {"wide": lambda c, i0, j0, s: wide_bands(c, i0, j0),
         "ragged": lambda c, i0, j0, s: ragged_bands(c, i0, j0, s),
         "qdb": lambda c, i0, j0, s: qdb_bands(c, i0, j0)}


def bits(x):
    return np.float32(x).tobytes()


def hb(hits):
    return [(i, j, bits(s), bits(b), m, r) for i, j, s, b, m, r in hits]


CASES = [(m, loc, p, kind, dense) for m in ("trna", "small2", "mb3") for loc in (False, True)
         for p in (2, 3, 4) for kind, dense in (("wide", True), ("ragged", False))] + \
        [("small0", True, 5, "qdb", True), ("cfg2", True, 4, "ragged", False), ("trna", False, 5, "wide", False)]


@pytest.mark.parametrize("case", CASES, ids=[f"{c[0]}-{'loc' if c[1] else 'glob'}-p{c[2]}-{c[3]}" for c in CASES])
def test_tr_scans_match_oracle(case):
    name, loc, pass_idx, kind, dense = case
    cm, g, l = models(name)
    cfg = l if loc else g
    seed = 71 + CASES.index(case)
    tt = tr_tables(cm, cfg, pass_idx, loc)
    tri = TrInputs(tt["lmesc"], tt["rmesc"], tt["pty"], tt["lpos"], tt["rpos"], tt["clen"], loc)
    sc = Scanner(cfg)
    for rep in range(2):
        f, i0, j0 = truncated_window(cm, cfg, pass_idx, seed * 10 + rep)
        b = BANDS[kind](cfg, i0, j0, seed + rep)
        valid = tr_valid(cfg.M, seed + rep, pass_idx, dense)
        for inside, fn in ((False, tr_cyk_scan_hb), (True, ftr_inside_scan_hb)):
            for cutoff, null3 in ((-10.0, True), (0.0, False)):
                ro = oracle.tr_hb_scan(cfg, inside, tt, valid, as_tuple(b), f, i0, j0, cutoff, null3, pass_idx,
                                       -5.0, loc)
                rg = fn(sc, tri, b, valid, f, i0, j0, cutoff, null3, pass_idx, -5.0)
                assert (bits(rg[1]), rg[2], rg[3], rg[4]) == (bits(ro[1]), ro[2], ro[3], ro[4]), (rep, inside, cutoff)
                assert hb(rg[0]) == hb(ro[0]), (rep, inside, cutoff)
    sc.close()


@pytest.mark.parametrize("semiring", [N.CYK_F32, N.INSIDE_F32])
def test_tr_batch_many_envelopes(semiring):
    cm, g, l = models("trna")
    loc = True
    sc = Scanner(l)
    frames, tasks, ref, off, nh = [], [], [], 0, 0
    pass_idx = 4
    tt = tr_tables(cm, l, pass_idx, loc)
    tri = TrInputs(tt["lmesc"], tt["rmesc"], tt["pty"], tt["lpos"], tt["rpos"], tt["clen"], loc)
    for q in range(20):
        f, i0, j0 = truncated_window(cm, l, pass_idx, 900 + q)
        b = (wide_bands, lambda c, a, z: ragged_bands(c, a, z, q))[q % 2](l, i0, j0)
        valid = tr_valid(l.M, q, pass_idx, q % 3 != 0)
        tasks.append((off, i0, j0, -5.0, -10.0, b, valid))
        ro = oracle.tr_hb_scan(l, semiring == N.INSIDE_F32, tt, valid, as_tuple(b), f, i0, j0, -10.0, True, pass_idx,
                               -5.0, loc)
        ref.append(ro)
        frames.append(f)
        off += len(f)
    got = tr_scan_hb_batch(sc, semiring, tri, pass_idx, True, np.concatenate(frames), tasks)
    for rg, ro in zip(got, ref):
        assert (bits(rg[1]), rg[2], rg[3], rg[4]) == (bits(ro[1]), ro[2], ro[3], ro[4])
        assert hb(rg[0]) == hb(ro[0])
        nh += len(ro[0])
    assert nh > 0
    sc.close()
