"""GPU Viterbi filter vs the oracle's vit_score_scalar: f32 score bits and
None (overflow) flags equal, on the reference test's own grid of random
profiles and sequences (src/p7_vitfilter.rs:603-635: every M around the
8-word vector boundary, L from 1 to 500, 8 profiles each, residue codes
0..15 including gap and IUPAC codes), plus long windows and a batch of
uneven windows in one launch."""
import numpy as np
import pytest

import oracle
from infernox_b200 import _native as N
from infernox_b200.p7 import VitFilter, vit_score

from p7_helpers import LS, Lcg, random_dsq, random_profile, reference_grid

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


def test_vit_matches_oracle_on_reference_grid():
    n = 0
    for p, seqs in reference_grid():
        buf, wins, offs, lens = frames_of(seqs)
        f = VitFilter(p)
        sc, ok = f.score_batch(buf, wins)
        rs, rok = oracle.vit_score_batch(p.M, p.mat, p.trans, buf, offs, lens)
        assert np.array_equal(ok, rok), p.M
        assert np.array_equal(sc[ok == 1].view(np.uint32), rs[rok == 1].view(np.uint32)), p.M
        f.close()
        n += len(seqs)
    assert n == 21 * 8 * len(LS)


@pytest.mark.parametrize("m", [33, 48, 97, 150, 190, 256, 257, 350, 1500])
def test_vit_long_windows_and_large_models(m):
    rng = Lcg(1000 + m)
    p = random_profile(rng, m)
    r = np.random.default_rng(m)
    seqs = []
    for l in (1, 999, 5000, 20000):
        d = np.zeros(l + 2, np.uint8)
        d[1:-1] = r.integers(0, 18, l)
        seqs.append(d)
    buf, wins, offs, lens = frames_of(seqs)
    f = VitFilter(p)
    sc, ok = f.score_batch(buf, wins)
    rs, rok = oracle.vit_score_batch(m, p.mat, p.trans, buf, offs, lens)
    assert np.array_equal(ok, rok)
    assert np.array_equal(sc[ok == 1].view(np.uint32), rs[rok == 1].view(np.uint32))
    # the single-window mirror of vit_score
    one = vit_score(f, buf[wins[1]["dsq_offset"]:], int(wins[1]["j0"]))
    assert (one is None) == (not rok[1])
    if one is not None:
        assert np.float32(one).tobytes() == rs[1].tobytes()
