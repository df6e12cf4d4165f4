"""Viterbi filter tables: the library's host build equals the oracle's
restatement of build_vit_filter on the reference test's random profiles
(no GPU: the filter is built with device = -1)."""
import ctypes as C

import numpy as np

import oracle
from infernox_b200 import _native as N
from infernox_b200.p7 import P7Profile

from p7_helpers import Lcg, MS, random_profile


def product_tables(p: P7Profile):
    mat = np.ascontiguousarray(p.mat, np.float32)
    trans = np.ascontiguousarray(p.trans, np.float32)
    prof = N.P7Profile(p.M, N.ptr(mat, C.c_float), N.ptr(trans, C.c_float))
    h = C.c_void_p()
    N.check(N.lib().cmgpu_vit_filter_build(C.byref(prof), -1, C.byref(h)))
    n = C.c_int32()
    N.lib().cmgpu_vit_filter_tables(h, None, 0, C.byref(n), None)
    tab = np.zeros(n.value, np.int16)
    sp = np.zeros(3, np.int16)
    N.check(N.lib().cmgpu_vit_filter_tables(h, tab.ctypes.data, n.value, C.byref(n), sp.ctypes.data))
    N.lib().cmgpu_vit_filter_free(h)
    return tab, sp


def test_vit_tables_match_oracle():
    rng = Lcg()
    for m in MS:
        for _ in range(2):
            p = random_profile(rng, m)
            t1, s1 = product_tables(p)
            t2, s2 = oracle.vit_tables(m, p.mat, p.trans)
            assert np.array_equal(t1, t2), m
            assert np.array_equal(s1, s2)
            assert s1[0] == 12000


def test_vit_oracle_sanity():
    """Scores are finite for residue sequences and -inf-free for L >= 1;
    longer random sequences do not score higher on average (a smoke check of
    the restated recursion)."""
    rng = Lcg(7)
    p = random_profile(rng, 40)
    bufs, offs, lens, off = [], [], [], 0
    for l in (10, 100, 1000):
        d = np.zeros(l + 2, np.uint8)
        d[1:-1] = np.random.default_rng(l).integers(0, 4, l)
        bufs.append(d)
        offs.append(off)
        lens.append(l)
        off += len(d)
    sc, ok = oracle.vit_score_batch(40, p.mat, p.trans, np.concatenate(bufs), offs, lens)
    assert ok.all() and np.isfinite(sc).all()


def test_oracle_sse_engine_equals_scalar_sweep():
    """The reference's own sse_matches_scalar property (src/p7_vitfilter.rs:
    603-635) on the oracle: its SSE2 striped engine (the timed CPU baseline)
    and its scalar sweep give the same score bits and overflow flags on the
    test's whole grid, and on long windows of larger models."""
    import numpy as np
    import oracle
    from p7_helpers import Lcg, random_profile, reference_grid
    n = 0
    for p, seqs in reference_grid():
        for d in seqs:
            L = len(d) - 2
            a = oracle.vit_score_batch(p.M, p.mat, p.trans, d, [0], [L])
            b = oracle.vit_score_batch(p.M, p.mat, p.trans, d, [0], [L], scalar=True)
            assert np.array_equal(a[1], b[1]) and a[0].tobytes() == b[0].tobytes(), (p.M, L)
            n += 1
    assert n == 1176
    for m in (97, 257, 1500):
        p = random_profile(Lcg(1000 + m), m)
        r = np.random.default_rng(m)
        d = np.full(5002, 255, np.uint8)
        d[1:-1] = r.integers(0, 18, 5000)
        a = oracle.vit_score_batch(m, p.mat, p.trans, d, [0], [5000])
        b = oracle.vit_score_batch(m, p.mat, p.trans, d, [0], [5000], scalar=True)
        assert np.array_equal(a[1], b[1]) and a[0].tobytes() == b[0].tobytes(), m
