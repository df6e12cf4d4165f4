"""CP9-style bands for the HMM-banded scanner tests.

* wide_bands: every state spans the whole envelope, as the reference's own
  test fixture builds them (src/cm_dpsearch_trunc.rs:2617-2661).
* rect_bands: per-state (i, j) rectangles turned into d-bands exactly as
  ij2d_bands does (src/cp9.rs:3815-3850): hdmin = max(j - imax + 1, sd),
  hdmax = j - imin + 1, rows with hdmax < sd empty (-1/-2), END rows 0/0.
  Rectangles are nested around seeded centres, so bands are narrow and
  some rows are empty, like real HMM bands.
* qdb_bands: every row of state v gets the QDB band [dmin1, dmax1] clipped
  to the envelope.
"""
import numpy as np

from infernox_b200 import synth
from infernox_b200.hb import Bands

from helpers import frame

E_ST, B_ST = 7, 8
EMIT = (1, 2, 3, 4, 5)  # MP, ML, MR, IL, IR


def sdelta(st):
    return 2 if st == 1 else (1 if st in (2, 3, 4, 5) else 0)


def wide_bands(cm, i0, j0):
    w = j0 - i0 + 1
    mins, maxs = [], []
    for v in range(cm.M):
        st = int(cm.sttype[v])
        dmax = np.minimum(np.arange(1, w + 1), w).astype(np.int32)
        if st == E_ST:
            mins.append(np.zeros(w, np.int32))
            maxs.append(np.zeros(w, np.int32))
        elif st in EMIT:
            mins.append(np.ones(w, np.int32))
            maxs.append(np.maximum(dmax, 1))
        else:
            mins.append(np.zeros(w, np.int32))
            maxs.append(dmax)
    return Bands.from_rows(np.full(cm.M, i0), np.full(cm.M, j0), mins, maxs)


def ij2d(cm, i0, j0, imin, imax, jmin, jmax):
    mins, maxs = [], []
    for v in range(cm.M):
        st = int(cm.sttype[v])
        n = max(0, jmax[v] - jmin[v] + 1)
        j = np.arange(jmin[v], jmin[v] + n)
        if st == E_ST:
            mins.append(np.zeros(n, np.int32))
            maxs.append(np.zeros(n, np.int32))
            continue
        dn = sdelta(st)
        hdn = j - imax[v] + 1
        hdx = j - imin[v] + 1
        lo = np.where(hdx < dn, -1, np.maximum(hdn, dn))
        hi = np.where(hdx < dn, -2, hdx)
        mins.append(lo.astype(np.int32))
        maxs.append(hi.astype(np.int32))
    return Bands.from_rows(jmin, jmax, mins, maxs)


def rect_bands(cm, i0, j0, seed, slack=6):
    """Seeded nested rectangles: state v's subsequence i..j sits around a
    centre span that shrinks from ROOT down the tree."""
    r = np.random.default_rng(seed)
    w = j0 - i0 + 1
    M = cm.M
    ci = np.zeros(M, np.int64)
    cj = np.zeros(M, np.int64)
    ci[0], cj[0] = i0 + r.integers(0, max(1, w // 8)), j0 - r.integers(0, max(1, w // 8))
    for v in range(M):
        st = int(cm.sttype[v])
        kids = []
        if st == B_ST:
            y, z = int(cm.cfirst[v]), int(cm.cnum[v])
            mid = (ci[v] + cj[v]) // 2 + r.integers(-3, 4)
            ci[y], cj[y] = ci[v], mid
            ci[z], cj[z] = mid + 1, cj[v]
            continue
        if st == E_ST:
            continue
        for yo in range(int(cm.cnum[v])):
            y = int(cm.cfirst[v]) + yo
            if y == v or y <= v:
                continue
            if ci[y] == 0 and cj[y] == 0:
                ci[y] = ci[v] + (1 if st in (1, 2) else 0)
                cj[y] = cj[v] - (1 if st in (1, 3) else 0)
    imin = np.clip(ci - r.integers(0, slack + 1, M), i0, j0).astype(np.int32)
    imax = np.clip(ci + r.integers(0, slack + 1, M), i0, j0).astype(np.int32)
    jmin = np.clip(cj - r.integers(0, slack + 1, M), i0, j0).astype(np.int32)
    jmax = np.clip(cj + r.integers(0, slack + 1, M), i0, j0).astype(np.int32)
    for v in range(M):
        if int(cm.sttype[v]) == E_ST:  # END: d = 0 cells, i = j + 1
            jmin[v] = max(i0 - 1, min(jmin[v], imin[v] - 1))
            jmax[v] = max(jmin[v], min(j0, jmax[v]))
    # a few states with no rows at all
    drop = r.random(M) < 0.03
    drop[0] = False
    jmax[drop] = jmin[drop] - 1
    return ij2d(cm, i0, j0, imin, imax, jmin, jmax)


def qdb_bands(cm, i0, j0):
    w = j0 - i0 + 1
    mins, maxs = [], []
    for v in range(cm.M):
        st = int(cm.sttype[v])
        jp = np.arange(w)
        if st == E_ST:
            mins.append(np.zeros(w, np.int32))
            maxs.append(np.zeros(w, np.int32))
            continue
        lo = np.maximum(int(cm.dmin1[v]), sdelta(st))
        hi = np.minimum(int(cm.dmax1[v]), jp + 1)
        mins.append(np.where(hi < lo, -1, lo).astype(np.int32))
        maxs.append(np.where(hi < lo, -2, hi).astype(np.int32))
    return Bands.from_rows(np.full(cm.M, i0), np.full(cm.M, j0), mins, maxs)


def as_tuple(b: Bands):
    return (b.jmin, b.jmax, b.hd_off, b.hdmin, b.hdmax)


def ragged_bands(cm, i0, j0, seed, trim=4):
    """wide bands with every row trimmed by a seeded amount at both ends
    (some rows become empty), and state j-ranges shortened at random."""
    r = np.random.default_rng(seed)
    b = wide_bands(cm, i0, j0)
    jmin, jmax = b.jmin.copy(), b.jmax.copy()
    mins, maxs = [], []
    for v in range(cm.M):
        st = int(cm.sttype[v])
        lo = b.hdmin[b.hd_off[v]: b.hd_off[v] + (b.jmax[v] - b.jmin[v] + 1)].copy()
        hi = b.hdmax[b.hd_off[v]: b.hd_off[v] + (b.jmax[v] - b.jmin[v] + 1)].copy()
        if st != E_ST and v != 0:
            lo = lo + r.integers(0, trim + 1, lo.size)
            hi = hi - r.integers(0, trim + 1, hi.size)
            cut0, cut1 = r.integers(0, 3), r.integers(0, 3)
            lo, hi = lo[cut0: lo.size - cut1], hi[cut0: hi.size - cut1]
            jmin[v] += cut0
            jmax[v] -= cut1
            empty = hi < lo
            lo[empty], hi[empty] = -1, -2
        mins.append(lo.astype(np.int32))
        maxs.append(hi.astype(np.int32))
    return Bands.from_rows(jmin, jmax, mins, maxs)


# ---- truncated-scan inputs ----------------------------------------------
def tr_tables(cm_s, cfg, pass_idx, local):
    """Per-pass truncated-scan inputs as a dict (hb.tr_inputs: the restated
    marginal emissions and truncated-begin penalties of the pass)."""
    from infernox_b200.hb import tr_inputs
    t = tr_inputs(cm_s, cfg, pass_idx, local)
    return {"lmesc": t.lmesc, "rmesc": t.rmesc, "pty": t.pty, "lpos": t.lpos, "rpos": t.rpos, "clen": t.clen,
            "ilmesc": t.ilmesc, "irmesc": t.irmesc, "ipty": t.ipty}


def tr_valid(M, seed, pass_idx, dense=True):
    """J/L/R/T validity per state: all true, or seeded sparse L/R/T."""
    r = np.random.default_rng(seed)
    j = np.ones(M, np.uint8)
    if dense:
        return j, np.ones(M, np.uint8), np.ones(M, np.uint8), np.ones(M, np.uint8)
    return j, (r.random(M) < 0.7).astype(np.uint8), (r.random(M) < 0.7).astype(np.uint8), \
        (r.random(M) < 0.5).astype(np.uint8)


def truncated_window(cm, cfg, pass_idx, seed, max_len=None, flank=30):
    """A sequence holding one sampled homolog and an envelope [i0, j0] that
    cuts it at the 5' end (pass 2), the 3' end (pass 3) or both (4, 5), with
    `flank` residues of background on an uncut side; at most max_len
    (default W) residues long."""
    rng = np.random.default_rng(seed)
    h = synth.emit(cm, rng)
    while len(h) < 20:
        h = synth.emit(cm, rng)
    n = len(h) + 2 * max(60, flank + 1)
    seq = synth.random_dsq(n, 0.5, rng)
    p = max(60, flank + 1)
    seq[p:p + len(h)] = h
    cut = max(3, len(h) // 4)
    i0, j0 = p + 1 - flank, p + len(h) + flank
    if pass_idx in (2, 4, 5):
        i0 = p + 1 + cut
    if pass_idx in (3, 4, 5):
        j0 = p + len(h) - cut
    j0 = min(j0, i0 + (max_len or cfg.W) - 1)
    return frame(seq), i0, j0
