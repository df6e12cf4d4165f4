"""GPU scanner vs the oracle: hits must be bit-identical.

CYK (f32 max-plus) and integer Inside (ILogsum) are both held to exact
equality of (i, j, score, bias) -- the kernel keeps the reference's
per-cell operand order, so no tolerance is needed.  Sizes are small enough
for the oracle to finish in seconds."""
import numpy as np
import pytest

import oracle
from infernox_b200 import scan
from infernox_b200.scan import CYK_F32, INSIDE_I32, KERNEL_LEVEL, KERNEL_SWEEP, NOQDB, QDB1, QDB2

from helpers import frame, models, oracle_cfg, planted_seq

pytestmark = pytest.mark.gpu

# both scan kernels must reproduce the oracle: the CTA level schedule and the
# warp node sweep
KERNELS = pytest.mark.parametrize("kernel", [KERNEL_LEVEL, KERNEL_SWEEP], ids=["level", "sweep"])


def scanner(cfg, kernel):
    s = scan.Scanner(cfg)
    s.set_kernel(kernel)
    return s


def hits_equal(gpu, ref):
    g = [(h.i, h.j, np.float32(h.score).tobytes(), np.float32(h.bias).tobytes()) for h in gpu]
    r = [(h[0], h[1], np.float32(h[2]).tobytes(), np.float32(h[3]).tobytes()) for h in ref]
    return g == r


CASES = [
    # model, local, semiring, band, n, cutoff, null3, degenerate
    ("trna", True, CYK_F32, QDB1, 2500, 0.0, True, 0.0),
    ("trna", False, CYK_F32, QDB1, 2500, 0.0, True, 0.0),
    ("trna", True, INSIDE_I32, QDB2, 2500, 0.0, True, 0.0),
    ("trna", False, INSIDE_I32, QDB2, 2500, -5.0, True, 0.0),
    ("trna", True, INSIDE_I32, NOQDB, 1500, 0.0, True, 0.0),
    ("trna", True, CYK_F32, NOQDB, 1500, 0.0, False, 0.0),
    ("small0", True, CYK_F32, QDB1, 3000, -2.0, True, 0.01),
    ("small0", True, INSIDE_I32, QDB2, 3000, -2.0, True, 0.01),
    ("small2", True, INSIDE_I32, NOQDB, 2000, 0.0, True, 0.0),
    ("small2", False, CYK_F32, QDB2, 2000, 0.0, False, 0.02),
    ("mb3", True, CYK_F32, QDB1, 2000, 0.0, True, 0.0),
    ("mb3", True, INSIDE_I32, QDB2, 2000, 0.0, True, 0.0),
    ("cfg2", True, INSIDE_I32, NOQDB, 1200, 0.0, True, 0.0),
    ("cfg2", True, CYK_F32, QDB1, 1200, 0.0, True, 0.0),
]


@KERNELS
@pytest.mark.parametrize("case", CASES, ids=lambda c: f"{c[0]}-{'L' if c[1] else 'G'}-s{c[2]}-b{c[3]}")
def test_generic_scan_matches_oracle(case, kernel):
    name, local, sr, band, n, cutoff, null3, degen = case
    cm, g, l = models(name)
    c = l if local else g
    seq = planted_seq(cm, n, 0.5, 3, seed=17 + CASES.index(case), degenerate=degen)
    dsq = frame(seq)
    # the oracle scans with its own tables; the GPU with the library's
    ref, _, _, _ = oracle.qdb_scan(oracle_cfg(name, local), sr, band, dsq, 1, n, cutoff, null3)
    s = scanner(c, kernel)
    got = s.generic_scan(sr, band, dsq, 1, n, cutoff, null3)
    assert s.stats()["kernel"] == kernel
    assert len(ref) > 0
    assert hits_equal(got, ref), (got[:5], ref[:5])


@KERNELS
@pytest.mark.parametrize("shape", [(0, 0, 0, 0), (0, 0, 200, 1), (0, 256, 200, 3), (2, 128, 1000, 2),
                                   (1, 512, 300, 8)])
def test_subchunked_windows_match(shape, kernel):
    """Forced small work items, several items per CTA: warm-up restarts and
    lane refills must not change any hit."""
    ctas, threads, chunk, lanes = shape
    cm, g, l = models("trna")
    n = 6000
    dsq = frame(planted_seq(cm, n, 0.45, 6, seed=7))
    s = scanner(l, kernel)
    s.set_shape(ctas_per_sm=ctas, threads=threads, chunk=chunk, lanes=lanes)
    for sr, band in ((CYK_F32, QDB1), (INSIDE_I32, QDB2)):
        ref, _, _, _ = oracle.qdb_scan(l, sr, band, dsq, 1, n, -3.0, True)
        got = s.generic_scan(sr, band, dsq, 1, n, -3.0, True)
        assert hits_equal(got, ref)


@KERNELS
def test_window_inside_frame(kernel):
    """Windows [i0, j0] strictly inside the frame (as envelopes are)."""
    cm, g, l = models("small2")
    n = 3000
    dsq = frame(planted_seq(cm, n, 0.5, 4, seed=9))
    s = scanner(l, kernel)
    for (i0, j0) in ((1, 1), (5, 40), (700, 1900), (2990, 3000), (1, 3000)):
        ref, _, _, _ = oracle.qdb_scan(l, INSIDE_I32, QDB2, dsq, i0, j0, -10.0, True)
        got = s.generic_scan(INSIDE_I32, QDB2, dsq, i0, j0, -10.0, True)
        assert hits_equal(got, ref), (i0, j0)


def test_cyk_filter_and_final_stage():
    """The --nohmm pair: QDB1 CYK envelopes, then QDB2 Inside per envelope."""
    cm, g, l = models("trna")
    n = 8000
    dsq = frame(planted_seq(cm, n, 0.5, 8, seed=3))
    s = scan.Scanner(l)
    env_ref = oracle.cyk_seq_filter(l, dsq, n, 5.0, True)
    env = s.cyk_seq_filter(dsq, n, 5.0, True)
    assert env == env_ref and len(env) > 0
    for nonbanded in (False, True):
        ref = oracle.final_stage_inside_opt(l, dsq, env, 8.0, True, nonbanded)
        got = s.final_stage_inside_opt(dsq, env, 8.0, True, nonbanded)
        assert hits_equal(got, ref)


@KERNELS
def test_batch_uneven_windows_match_per_window(kernel):
    """Many windows of uneven length in one launch == each window alone."""
    cm, g, l = models("small2")
    rng = np.random.default_rng(42)
    lens = np.clip(rng.lognormal(np.log(300), 1.0, 40).astype(int), 1, 3000)
    frames, wins, off = [], [], 0
    for k, L in enumerate(lens):
        f = frame(planted_seq(cm, int(L), 0.45, 1 if L > 200 else 0, seed=100 + k))
        frames.append(f)
        wins.append((off, 1, int(L)))
        off += len(f)
    buf = np.concatenate(frames)
    W = np.array(wins, dtype=[("dsq_offset", np.int64), ("i0", np.int32), ("j0", np.int32)])
    s = scanner(l, kernel)
    for sr, band in ((INSIDE_I32, NOQDB), (CYK_F32, QDB1)):
        got = s.scan_batch(sr, band, buf, W, 0.0, True)
        plain = s.scan_batch(sr, band, buf, W, 0.0, True, plain=True)
        assert np.array_equal(got, plain)
        k = 0
        for w, (o, i0, j0) in enumerate(wins):
            f = buf[o:o + j0 + 2]
            ref, _, _, _ = oracle.qdb_scan(l, sr, band, f, i0, j0, 0.0, True)
            mine = got[got["win"] == w]
            assert [(int(h["i"]), int(h["j"]), h["score"].tobytes(), h["bias"].tobytes()) for h in mine] == \
                   [(r[0], r[1], np.float32(r[2]).tobytes(), np.float32(r[3]).tobytes()) for r in ref]
            k += len(mine)
        assert k == len(got)


def test_counts_match_oracle_counters():
    cm, g, l = models("mb3")
    n = 1500
    dsq = frame(planted_seq(cm, n, 0.5, 1, seed=5))
    s = scan.Scanner(l)
    for sr, band in ((CYK_F32, QDB1), (INSIDE_I32, NOQDB)):
        _, _, cells, terms = oracle.qdb_scan(l, sr, band, dsq, 1, n, 0.0, False)
        s.generic_scan(sr, band, dsq, 1, n, 0.0, False)
        st = s.stats()
        assert st["cells"] == cells and st["terms"] == terms
        assert st["kernel_launches"] >= 1


CELL_CASES = [
    ("trna", True, INSIDE_I32, QDB2), ("trna", False, INSIDE_I32, QDB2),
    ("trna", True, INSIDE_I32, NOQDB), ("small0", True, INSIDE_I32, QDB2),
    ("trna", True, CYK_F32, QDB1), ("mb3", False, INSIDE_I32, NOQDB),
]


@KERNELS
@pytest.mark.parametrize("case", CELL_CASES, ids=lambda c: f"{c[0]}-{'L' if c[1] else 'G'}-s{c[2]}-b{c[3]}")
def test_all_cells_match_oracle(case, kernel):
    """Every ROOT cell (j, d) above a very low cutoff, bit for bit."""
    name, local, sr, band = case
    cm, g, l = models(name)
    c = l if local else g
    n = 400
    dsq = frame(planted_seq(cm, n, 0.5, 1, seed=55))
    _, ref, _, _ = oracle.qdb_scan(c, sr, band, dsq, 1, n, -1e30, False, want_cands=True)
    got = scanner(c, kernel).scan_cells(sr, band, dsq, 1, n, -1e30)
    rmap = {(j, d): s for j, d, s in ref}
    gmap = {(j, d): s for j, d, s in got}
    bad = [(k, gmap.get(k), rmap.get(k)) for k in sorted(set(rmap) | set(gmap))
           if np.float32(gmap.get(k, np.nan)).tobytes() != np.float32(rmap.get(k, np.nan)).tobytes()]
    assert not bad, (len(bad), len(ref), bad[:8])
