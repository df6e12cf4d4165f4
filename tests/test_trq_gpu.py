"""GPU truncated QDB / non-banded scanner vs the oracle (generic_tr_scan
restated: ref_tr_cyk_scan and ref_itr_inside_scan), through the C ABI.

Equal bits of vsc_root with its marginal mode, of the full-window score
bsc_full, and equal reported hits (i, j, score bits, bias bits, mode, entry
state) after overlap removal, for TrCYK (f32) and the integer TrInside, in
the truncated passes 5'-only, 3'-only, 5'-and-3' and 5'-and-3'-any, global
and local truncation rules, non-banded and with both QDB band sets, on
windows that cut a sampled homolog at the 5' end, the 3' end or both; on
windows longer than W (the BEGL ring wraps, jrow saturates) and windows
starting at residue 1 (bsc_full is set); then a batch of windows of mixed
lengths, an empty one among them, in one call.
"""
import numpy as np
import pytest

import oracle
from infernox_b200 import _native as N
from infernox_b200.hb import TrInputs, ref_itr_inside_scan, ref_tr_cyk_scan, tr_qdb_scan_batch
from infernox_b200.scan import Scanner

from hb_helpers import tr_tables, truncated_window
from helpers import frame, models

pytestmark = pytest.mark.gpu


def bits(x):
    return np.float32(x).tobytes()


def hb(hits):
    return [(i, j, bits(s), bits(b), m, r) for i, j, s, b, m, r in hits]


def tri_of(tt, loc):
    return TrInputs(tt["lmesc"], tt["rmesc"], tt["pty"], tt["lpos"], tt["rpos"], tt["clen"], loc,
                    tt["ilmesc"], tt["irmesc"], tt["ipty"])


def check(cfg, sc, tt, loc, f, i0, j0, qdb, pass_idx, cutoff, null3, what):
    for inside, fn in ((False, ref_tr_cyk_scan), (True, ref_itr_inside_scan)):
        ro = oracle.trq_scan(cfg, inside, tt, f, i0, j0, cutoff, null3, qdb, pass_idx, loc)
        go = fn(sc, tri_of(tt, loc), f, i0, j0, cutoff, qdb, null3, pass_idx)
        tag = (what, "inside" if inside else "cyk", qdb, pass_idx, cutoff, null3)
        assert bits(go[1]) == bits(ro[1]) and go[2] == ro[2], (tag, go[1:], ro[1:])
        assert bits(go[3]) == bits(ro[3]), (tag, go[3], ro[3])
        assert hb(go[0]) == hb(ro[0]), (tag, go[0][:4], ro[0][:4])


CASES = [(m, loc, p, qdb) for m in ("trna", "small2", "mb3") for loc in (False, True)
         for p in (2, 3, 4) for qdb in (N.NOQDB, N.QDB1)] + \
        [("small0", True, 5, N.QDB2), ("small0", False, 4, N.NOQDB), ("cfg2", True, 4, N.QDB2),
         ("cfg2", False, 2, N.NOQDB), ("trna", True, 5, N.QDB2), ("mb3", False, 5, N.NOQDB)]


@pytest.mark.parametrize("case", CASES, ids=[f"{c[0]}-{'loc' if c[1] else 'glob'}-p{c[2]}-q{c[3]}" for c in CASES])
def test_trq_scans_match_oracle(case):
    name, loc, pass_idx, qdb = case
    cm, g, l = models(name)
    cfg = l if loc else g
    seed = 301 + CASES.index(case)
    tt = tr_tables(cm, cfg, pass_idx, loc)
    sc = Scanner(cfg)
    f, i0, j0 = truncated_window(cm, cfg, pass_idx, seed)
    for cutoff, null3 in ((-10.0, True), (0.0, False)):
        check(cfg, sc, tt, loc, f, i0, j0, qdb, pass_idx, cutoff, null3, "window")


@pytest.mark.parametrize("name", ["trna", "small0", "mb3"])
def test_trq_long_and_leading_windows(name):
    """Windows longer than W (ring wrap of the BEGL decks, saturated rows) and
    windows that start at residue 1 with j0 <= W (bsc_full defined)."""
    cm, g, l = models(name)
    for loc, cfg in ((False, g), (True, l)):
        sc = Scanner(cfg)
        for pass_idx in (2, 4):
            tt = tr_tables(cm, cfg, pass_idx, loc)
            f, i0, j0 = truncated_window(cm, cfg, 3, 17 + pass_idx, max_len=cfg.W + 45, flank=60)
            check(cfg, sc, tt, loc, f, i0, j0, N.NOQDB, pass_idx, -5.0, True, "long")
            check(cfg, sc, tt, loc, f, i0, j0, N.QDB1, pass_idx, -5.0, False, "long")
            L = min(cfg.W, (f.size - 2))
            check(cfg, sc, tt, loc, f, 1, L - 3, N.NOQDB, pass_idx, -5.0, True, "lead")


def test_trq_batch_matches_single_windows():
    cm, g, l = models("mb3")
    sc = Scanner(l)
    pass_idx = 4
    tt = tr_tables(cm, l, pass_idx, True)
    tri = tri_of(tt, True)
    frames, wins, off = [], [], 0
    for q in range(9):
        f, i0, j0 = truncated_window(cm, l, 2 + q % 3, 900 + q, max_len=(l.W + 30) if q % 4 == 0 else None)
        if q == 5:
            i0, j0 = 40, 39  # empty
        frames.append(f)
        wins.append((off, i0, j0))
        off += f.size
    buf = np.concatenate(frames)
    w = np.array(wins, N.WINDOW_DTYPE)
    for semiring, inside in ((N.CYK_F32, False), (N.INSIDE_I32, True)):
        res = tr_qdb_scan_batch(sc, semiring, N.QDB1, tri, pass_idx, True, buf, w, -8.0)
        for q, (f, (o, i0, j0)) in enumerate(zip(frames, wins)):
            ro = oracle.trq_scan(l, inside, tt, f, i0, j0, -8.0, True, N.QDB1, pass_idx, True)
            go = res[q]
            assert bits(go[1]) == bits(ro[1]) and go[2] == ro[2] and bits(go[3]) == bits(ro[3]), (q, go[1:], ro[1:])
            assert hb(go[0]) == hb(ro[0]), (q, inside)


def test_trq_rejects_bad_inputs():
    cm, g, l = models("small2")
    sc = Scanner(g)
    tt = tr_tables(cm, g, 2, False)
    f, i0, j0 = truncated_window(cm, g, 2, 5)
    no_int = TrInputs(tt["lmesc"], tt["rmesc"], tt["pty"], tt["lpos"], tt["rpos"], tt["clen"], False)
    with pytest.raises(N.CmgpuError):  # the integer scan needs the integer tables
        ref_itr_inside_scan(sc, no_int, f, i0, j0, 0.0, N.NOQDB, False, 2)
    with pytest.raises(N.CmgpuError):  # no such band set
        ref_tr_cyk_scan(sc, tri_of(tt, False), f, i0, j0, 0.0, 3, False, 2)
    with pytest.raises(N.CmgpuError):  # window beyond the sequence
        ref_tr_cyk_scan(sc, tri_of(tt, False), f, i0, f.size, 0.0, N.NOQDB, False, 2)
    bad = f.copy()
    bad[i0 + 1] = 40
    with pytest.raises(ValueError):
        ref_tr_cyk_scan(sc, tri_of(tt, False), bad, i0, j0, 0.0, N.NOQDB, False, 2)


@pytest.mark.parametrize("name,loc,qdb", [("trna", True, N.NOQDB), ("small2", False, N.QDB2), ("small0", True, N.QDB1)])
def test_trq_edge_windows_and_passes(name, loc, qdb):
    """Every truncated pass, windows of 1 and 2 residues, IUPAC degenerate
    residues in the window, and a model without bifurcations (small0); the
    standard pass 1 and pass 6, which the reference's truncated scanners do
    not take (pty_idx_for_pass(..).expect), are refused."""
    from helpers import planted_seq
    cm, g, l = models(name)
    cfg = l if loc else g
    sc = Scanner(cfg)
    f = frame(planted_seq(cm, 400, 0.45, 2, seed=31, degenerate=0.1))
    for pass_idx in (2, 3, 4, 5):
        tt = tr_tables(cm, cfg, pass_idx, loc)
        for i0, j0 in ((50, 50), (50, 51), (10, 10 + cfg.W // 2), (100, 100 + cfg.W + 20)):
            check(cfg, sc, tt, loc, f, i0, j0, qdb, pass_idx, -20.0, True, ("edge", i0, j0))
    tt = tr_tables(cm, cfg, 4, loc)
    for bad in (1, 6):
        with pytest.raises(N.CmgpuError, match="truncated pass") as ei:
            ref_tr_cyk_scan(sc, tri_of(tt, loc), f, 50, 90, -20.0, qdb, True, bad)
        assert ei.value.rc == -1  # CMGPU_EINVAL


def test_trq_column_wait_times_out_and_reports():
    """Failure detection without a GPU fault: the warp of one column never
    publishes its progress (the test hook), the next column's bounded wait
    runs out, the call fails with CMGPU_ETIMEOUT, and the model scans
    correctly afterwards."""
    cm, g, l = models("small2")
    sc = Scanner(l)
    tt = tr_tables(cm, l, 4, True)
    f, i0, j0 = truncated_window(cm, l, 4, 77, max_len=l.W + 10, flank=60)
    assert j0 - i0 + 1 > 12
    N.check(N.lib().cmgpu_tr_qdb_inject_stall(sc._model, 3))
    with pytest.raises(N.CmgpuError, match="timed out") as ei:
        ref_tr_cyk_scan(sc, tri_of(tt, True), f, i0, j0, -5.0, N.NOQDB, True, 4)
    assert ei.value.rc == -6  # CMGPU_ETIMEOUT
    check(l, sc, tt, True, f, i0, j0, N.NOQDB, 4, -5.0, True, "after a timeout")
