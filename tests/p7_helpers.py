"""Random P7 filter profiles and sequences drawn exactly as the reference's
Viterbi test draws them (src/p7_vitfilter.rs:547-600): the same LCG
constants and seed, uniform draws in [0.05, 1.05), per-state normalisation,
residue codes 0..15, and the same M / L grids (:611-612)."""
import numpy as np

from infernox_b200.p7 import P7Profile

MASK64 = (1 << 64) - 1
MS = [1, 2, 3, 7, 8, 9, 15, 16, 17, 23, 24, 25, 31, 32, 40, 63, 64, 65, 100, 128, 200]
LS = [1, 2, 5, 17, 50, 200, 500]


class Lcg:
    def __init__(self, seed=0x123456789ABCDEF0):
        self.s = seed

    def next_u32(self):
        self.s = (self.s * 6364136223846793005 + 1442695040888963407) & MASK64
        return self.s >> 33

    def unit(self):
        # 0.05 + (next_u32 as f32 / u32::MAX as f32), all in f32
        return np.float32(np.float32(0.05) + np.float32(np.float32(self.next_u32()) / np.float32(4294967295.0)))


def random_profile(rng: Lcg, m: int) -> P7Profile:
    mat = np.zeros((m + 1, 4), np.float32)
    trans = np.zeros((m + 1, 7), np.float32)
    for k in range(1, m + 1):
        e = [rng.unit() for _ in range(4)]
        s = np.float32(0.0)
        for x in e:
            s = np.float32(s + x)
        mat[k] = [np.float32(x / s) for x in e]
    for k in range(m + 1):
        mm, mi, md = rng.unit(), rng.unit(), rng.unit()
        ms = np.float32(np.float32(mm + mi) + md)
        im, ii = rng.unit(), rng.unit()
        is_ = np.float32(im + ii)
        dm, dd = rng.unit(), rng.unit()
        ds = np.float32(dm + dd)
        trans[k] = [mm / ms, mi / ms, md / ms, im / is_, ii / is_, dm / ds, dd / ds]
    return P7Profile(m, mat, trans)


def random_dsq(rng: Lcg, l: int) -> np.ndarray:
    d = np.zeros(l + 2, np.uint8)
    for i in range(1, l + 1):
        d[i] = rng.next_u32() % 16
    return d


def reference_grid(reps=8):
    """(profile, [dsq for each L]) in the reference test's draw order."""
    rng = Lcg()
    out = []
    for m in MS:
        for _ in range(reps):
            p = random_profile(rng, m)
            seqs = [random_dsq(rng, l) for l in LS]
            out.append((p, seqs))
    return out
