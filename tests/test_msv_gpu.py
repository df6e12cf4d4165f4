"""GPU MSV score and SSV windows vs the oracle, through the C ABI.

* msv_score / msv_score_reconfig (src/cm_pipeline.rs:402-452): f32 score bits
  and None (8-bit overflow) flags equal, on the reference Viterbi test's grid
  of random profiles and sequences, and on planted sequences that overflow.
* ssv_diagonals (:521-717) and f1_msv_windows (:842): every raw diagonal
  (target start, model length, model end, score bits) and every final window
  equal, over many chunks per call, with trigger clusters (triggers within
  M rows of an earlier reset), dense triggers that overflow the per-segment
  candidate slots, IUPAC residues, chunks inside frames and empty chunks.
"""
import numpy as np
import pytest

import oracle
from infernox_b200 import _native as N
from infernox_b200.p7 import MsvFilter, f1_msv_windows, msv_score, msv_score_reconfig

from p7_helpers import LS, peaked_profile, planted_frame, reference_grid

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


def same_f32(a, b):
    return np.array_equal(np.asarray(a, np.float32).view(np.uint32), np.asarray(b, np.float32).view(np.uint32))


@pytest.mark.parametrize("reconfig", [False, True])
def test_msv_score_matches_oracle_on_reference_grid(reconfig):
    n = 0
    for p, seqs in reference_grid(reps=3):
        buf, wins, offs, lens = frames_of(seqs)
        wl = [max(1, 3 * l // 2) for l in lens] if reconfig else None
        f = MsvFilter(p, 200)
        sc, ok = f.score_batch(buf, wins, wl)
        rs, rok = oracle.msv_score_batch(p.M, p.mat, p.trans, 200, buf, offs, lens, wl)
        assert np.array_equal(ok, rok), p.M
        assert same_f32(sc[ok == 1], rs[rok == 1]), p.M
        f.close()
        n += len(seqs)
    assert n == 21 * 3 * len(LS)


@pytest.mark.parametrize("m", [40, 100, 350, 1500])
def test_msv_score_overflow_and_long_windows(m):
    p, cons = peaked_profile(50 + m, m)
    seqs = [planted_frame(60 + q, l, cons, nplant) for q, (l, nplant) in
            enumerate([(300, 0), (5000, 0), (5000, 3), (20000, 6), (1, 0), (2000, 1)])]
    buf, wins, offs, lens = frames_of(seqs)
    f = MsvFilter(p, int(1.25 * m))
    sc, ok = f.score_batch(buf, wins)
    rs, rok = oracle.msv_score_batch(m, p.mat, p.trans, int(1.25 * m), buf, offs, lens)
    assert np.array_equal(ok, rok)
    assert same_f32(sc[ok == 1], rs[rok == 1])
    assert (rok == 0).any() and (rok == 1).any()  # both outcomes exercised
    # the single-window mirrors
    a = buf[offs[1]: offs[1] + lens[1] + 2]
    one = msv_score(f, a, lens[1])
    assert one is not None and np.float32(one).tobytes() == rs[1].tobytes()
    rec = msv_score_reconfig(f, a, lens[1], 777)
    rr, rrok = oracle.msv_score_batch(m, p.mat, p.trans, int(1.25 * m), a, [0], [lens[1]], [777])
    assert rrok[0] and np.float32(rec).tobytes() == rr[0].tobytes()


SSV_CASES = [
    # (m, lmmu, f1, chunk length, chunks, plants per chunk)
    (100, -8.0, 0.02, 20000, 3, 8),
    (100, -8.0, 0.35, 20000, 3, 8),
    (40, -6.0, 0.9, 20000, 3, 8),      # dense triggers: candidate-slot overflow and retry
    (350, -10.0, 0.02, 20000, 3, 8),   # triggers within M rows of a reset
    (1000, -12.0, 0.02, 30000, 2, 10),
    (7, -4.0, 0.5, 5000, 4, 20),
    (1, -2.0, 0.9, 3000, 2, 0),
    (2048, -12.0, 0.05, 40000, 1, 10),
]


@pytest.mark.parametrize("case", SSV_CASES, ids=[f"M{c[0]}_f1{c[2]}" for c in SSV_CASES])
def test_ssv_diagonals_and_f1_windows_match_oracle(case):
    m, mmu, f1, l, nch, nplant = case
    p, cons = peaked_profile(11 + m, m)
    seqs = [planted_frame(100 + q, l, cons, nplant) for q in range(nch)]
    buf, wins, offs, lens = frames_of(seqs)
    maxl, cmw = int(1.25 * m), max(1, int(1.2 * m))
    ow, ows, oraw, orsc = oracle.f1_msv_windows(m, p.mat, p.trans, maxl, mmu, 0.69, buf, offs, lens, f1, cmw)
    assert len(oraw) > 0 or m == 1
    f = MsvFilter(p, maxl, mmu, 0.69)
    raw = f.ssv_diagonals_batch(buf, wins, f1)
    got = np.stack([raw["chunk"], raw["n"], raw["length"], raw["k"]], 1) if len(raw) else np.zeros((0, 4), np.int64)
    assert np.array_equal(got, oraw)
    assert same_f32(raw["score"], orsc)
    w = f.f1_windows_batch(buf, wins, f1, cmw)
    gw = np.stack([w["chunk"], w["start"], w["end"]], 1) if len(w) else np.zeros((0, 3), np.int64)
    assert np.array_equal(gw, ow)
    assert same_f32(w["score"], ows)
    ms, cells, launches = f.stats()
    assert cells >= sum(lens) * m and launches >= 2
    f.close()


def test_ssv_chunks_inside_frames_and_empty_chunks():
    m = 120
    p, cons = peaked_profile(5, m)
    fr = planted_frame(9, 30000, cons, 12)
    # three chunks cut from one frame, overlapping, plus an empty one
    wins = np.array([(0, 1, 12000), (0, 9001, 30000), (0, 500, 499), (0, 20000, 20050)], N.WINDOW_DTYPE)
    f = MsvFilter(p, 150, -8.0, 0.69)
    got = f.f1_windows_batch(fr, wins, 0.1, 144)
    # the oracle sees each chunk as its own frame starting one residue early
    offs = [int(w["dsq_offset"]) + int(w["i0"]) - 1 for w in wins]
    lens = [int(w["j0"]) - int(w["i0"]) + 1 for w in wins]
    ow, ows, _, _ = oracle.f1_msv_windows(m, p.mat, p.trans, 150, -8.0, 0.69, fr, offs, lens, 0.1, 144)
    gw = np.stack([got["chunk"], got["start"], got["end"]], 1)
    assert np.array_equal(gw, ow) and same_f32(got["score"], ows)
    assert len(ow) > 0 and not (gw[:, 0] == 2).any()
    # the single-chunk mirror of f1_msv_windows
    a = fr[: 12000 + 2].copy()
    a[-1] = 255
    one = f1_msv_windows(f, a, 12000, 0.1, 144)
    sel = ow[ow[:, 0] == 0]
    assert [(s, e) for s, e, _ in one] == [(int(r[1]), int(r[2])) for r in sel]


def test_ssv_rejects_bad_residues_and_windows():
    p, cons = peaked_profile(5, 50)
    f = MsvFilter(p, 60, -8.0, 0.69)
    fr = planted_frame(1, 1000, cons, 1)
    fr[10] = 18
    with pytest.raises(N.CmgpuError):
        f.f1_windows_batch(fr, np.array([(0, 1, 1000)], N.WINDOW_DTYPE), 0.1, 60)
    with pytest.raises(N.CmgpuError):
        f.f1_windows_batch(fr, np.array([(0, 1, 5000)], N.WINDOW_DTYPE), 0.1, 60)
