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


def peaked_profile(seed: int, m: int, peak: float = 0.85):
    """A profile with one strong residue per match position (so SSV/MSV
    diagonals along planted consensus runs score high) and its consensus."""
    r = np.random.default_rng(seed)
    mat = np.zeros((m + 1, 4), np.float32)
    cons = r.integers(0, 4, m + 1)
    for k in range(1, m + 1):
        v = r.uniform(0.02, 0.1, 4)
        v[cons[k]] = 0.0
        v = v / v.sum() * (1.0 - peak)
        v[cons[k]] = peak
        mat[k] = v.astype(np.float32)
    trans = np.zeros((m + 1, 7), np.float32)
    for k in range(m + 1):
        mi, md = r.uniform(0.01, 0.08, 2)
        ii = r.uniform(0.2, 0.6)
        dd = r.uniform(0.1, 0.5)
        trans[k] = [1 - mi - md, mi, md, 1 - ii, ii, 1 - dd, dd]
    return P7Profile(m, mat, trans), cons


def planted_frame(seed: int, l: int, cons, nplant: int, mut: float = 0.1, iupac: float = 0.002):
    """[255, residues..., 255] of i.i.d. codes with nplant consensus runs."""
    r = np.random.default_rng(seed)
    d = np.full(l + 2, 255, np.uint8)
    d[1:-1] = r.integers(0, 4, l)
    ambig = r.random(l) < iupac
    d[1:-1][ambig] = r.integers(4, 16, int(ambig.sum()))
    m = len(cons) - 1
    for _ in range(nplant):
        k0 = int(r.integers(1, max(2, m // 2)))
        k1 = int(min(m, k0 + r.integers(max(2, m // 4), m + 1)))
        run = np.array(cons[k0:k1 + 1], np.uint8)
        flip = r.random(len(run)) < mut
        run[flip] = r.integers(0, 4, int(flip.sum()))
        if len(run) >= l:
            continue
        p = int(r.integers(1, l - len(run) + 1))
        d[p:p + len(run)] = run
    return d
