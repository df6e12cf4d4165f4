"""cmcalibrate's host parts, no GPU: the random genomic sequences against the
reference's own known answer (rng_sample_matches_c, src/cm_calibrate.rs:
1253-1268, generated by C Infernal), the library's generator against the
oracle's restatement, and the tail fit (fit_histogram + set_exp_info)
against the oracle bit for bit, with the reference's error cases."""
import json
import os

import numpy as np
import pytest

import oracle
from infernox_b200 import calibrate as cal

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "genomic_kat.json")


def test_generator_matches_reference_known_answer():
    kat = json.load(open(GOLDEN))
    L, seqs = kat["L"], kat["sequences"]
    for frames in (cal.sample_genomic_sequences(kat["seed"], L, len(seqs)),
                   oracle.genomic_sample(kat["seed"], L, len(seqs))):
        for s, want in enumerate(seqs):
            f = frames[s * (L + 2):(s + 1) * (L + 2)]
            assert f[0] == 255 and f[-1] == 255
            assert "".join(str(int(x)) for x in f[1:-1]) == want


@pytest.mark.parametrize("seed,L,n", [(181, 10000, 3), (1, 777, 5), (4242, 1, 9), (0, 50, 2)])
def test_generator_matches_oracle(seed, L, n):
    a = cal.sample_genomic_sequences(seed, L, n)
    b = oracle.genomic_sample(seed, L, n)
    assert np.array_equal(a, b)


def test_generator_composition_is_genomic():
    """The five-state HMM's long runs of AT- and GC-rich states show as a
    composition well away from uniform in 10 kb windows."""
    f = cal.sample_genomic_sequences(181, 10000, 8).reshape(8, 10002)[:, 1:-1]
    gc = ((f == 1) | (f == 2)).mean(axis=1)
    assert (f <= 3).all()
    assert gc.std() > 0.02


def same(a, b):
    return all(np.float64(a[k]).tobytes() == np.float64(b[k]).tobytes() for k in ("mu", "mu_orig", "tailp", "dbsize")) \
        and np.float64(a["lambda_"]).tobytes() == np.float64(b["lambda"]).tobytes() and a["nrandhits"] == b["nrandhits"]


@pytest.mark.parametrize("mode", [0, 1, 2, 3])
@pytest.mark.parametrize("n", [40, 5000, 123457])
def test_exp_fit_matches_oracle(mode, n):
    rng = np.random.default_rng(n + mode)
    scores = (rng.gumbel(-20.0, 3.0, n) + (rng.random(n) < 0.01) * -987654.0).astype(np.float32)
    n_seqs = max(1, n // 5000)
    mine = cal.fit_histogram(scores, mode, n_seqs, 10000, 250, 750, None, 10000.0 * n_seqs)
    ref = oracle.exp_fit(scores, mode, n_seqs, 10000, 250, 750, 0.0, 10000.0 * n_seqs)
    assert ref is not None
    assert same(mine, ref), (mine, ref)
    # fixed tail mass
    mine = cal.fit_histogram(scores, mode, n_seqs, 10000, tailp=0.25, dbsize=1.0)
    ref = oracle.exp_fit(scores, mode, n_seqs, 10000, 250, 750, 0.25, 1.0)
    assert same(mine, ref)


def test_exp_fit_errors_as_reference():
    from infernox_b200 import _native as N
    s = np.linspace(-30, 10, 100).astype(np.float32)
    # tailn too large: more hits wanted than the histogram holds
    with pytest.raises(N.CmgpuError):
        cal.fit_histogram(s, 2, 100, 10000)
    assert oracle.exp_fit(s, 2, 100, 10000) is None
    # too few points in the tail
    with pytest.raises(N.CmgpuError):
        cal.fit_histogram(s, 0, 1, 10000, tailp=0.015)
    assert oracle.exp_fit(s, 0, 1, 10000, tailp=0.015) is None
    # a non-finite score fails the histogram
    bad = s.copy()
    bad[3] = np.inf
    with pytest.raises(N.CmgpuError):
        cal.fit_histogram(bad, 0, 1, 10000, tailp=0.5)
    assert oracle.exp_fit(bad, 0, 1, 10000, tailp=0.5) is None


def test_n_sequences_rounds_like_reference():
    assert cal.n_sequences(cal.CalibrateConfig()) == 160
    assert cal.n_sequences(cal.CalibrateConfig(l_mb=0.02)) == 2
    assert cal.n_sequences(cal.CalibrateConfig(l_mb=0.005)) == 1
    assert cal.n_sequences(cal.CalibrateConfig(l_mb=0.004)) == 0


def _fit_complete(xs):
    """esl_exp_FitComplete (src/easel/exponential.rs:67-89): mu = the lowest
    tail score, lambda = 1 / mean(x - mu), summed in tail order."""
    mu = min(xs)
    mean = 0.0
    for x in xs:
        mean += x - mu
    return mu, 1.0 / (mean / len(xs))


def test_tail_fit_matches_the_libeasel_probe():
    """The reference's test_cmcalibrate_sequence: the tail of mass 0.5 of its
    20 scores fitted by esl_exp_FitComplete gives the mu and lambda it pins to
    a probe of C libeasel.  The formula reproduces them bit for bit on those
    (double) scores, and the library's tail fit -- fed the same scores as the
    floats cmcalibrate's scans produce -- returns that formula's value on the
    floats, in every exp mode."""
    kat = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "histogram_kat.json")))
    s64 = kat["scores"]
    n = int(len(s64) * kat["tail_mass"])
    mu, lam = _fit_complete(sorted(s64)[len(s64) - n:])
    assert mu == float(kat["mu"]) and lam == float(kat["lambda"])
    s32 = np.asarray(s64, np.float32)
    fmu, flam = _fit_complete(sorted(float(x) for x in s32)[len(s64) - n:])
    for mode in range(4):
        r = cal.fit_histogram(s32, mode, 1, 10000, tailp=kat["tail_mass"], dbsize=1.0)
        assert np.float64(r["mu_orig"]).tobytes() == np.float64(fmu).tobytes()
        assert np.float64(r["lambda_"]).tobytes() == np.float64(flam).tobytes()
        assert r["nrandhits"] == len(s64)
