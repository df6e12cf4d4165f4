"""cmcalibrate on the GPU against the oracle.

collect_scores's scan (cutoff -inf, local begins compared in bit scores):
the kept hits of every window -- (i, j, score bits, bias bits) in order --
equal the oracle's restatement of cmcalibrate's generic_scan, in all four
exp modes, QDB and full bands, with and without null3, on random genomic
sequences from the reference's generator and on sequences holding homologs.
The oracle scans tables from its own builders (oracle/prep_oracle.c).
Then the whole calibration (cmgpu_calibrate) equals the oracle's
generator + scan + fit, bit for bit in every fitted parameter."""
import numpy as np
import pytest

import oracle
from infernox_b200 import _native as N
from infernox_b200 import calibrate as cal
from infernox_b200.model import ConfiguredCM
from infernox_b200.scan import Scanner

from helpers import frame, models, planted_seq

pytestmark = pytest.mark.gpu


def oracle_calib_cfg(cm, local, W, beta, nonbanded=False):
    t = oracle.prep_configure(cm, local, W, beta, beta)
    c = ConfiguredCM(
        name=cm.name, M=cm.M, W=t["W"], flags=t["flags"], clen=cm.clen,
        sttype=np.ascontiguousarray(cm.st.sttype, np.int8), stid=np.ascontiguousarray(cm.st.stid, np.int8),
        cfirst=np.ascontiguousarray(cm.st.cfirst, np.int32), cnum=np.ascontiguousarray(cm.st.cnum, np.int32),
        el_selfsc=t["el_selfsc"], iel_selfsc=t["iel_selfsc"], null=np.asarray(cm.null, np.float32),
        n3_omega=float(np.float32(cm.n3_omega)),
        **{k: t[k] for k in ("tsc", "oesc", "endsc", "beginsc", "itsc", "ioesc", "iendsc", "ibeginsc",
                             "dmin1", "dmax1", "dmin2", "dmax2", "t_local")})
    if nonbanded:
        c.dmin1[:] = 0
        c.dmin2[:] = 0
        c.dmax1[:] = c.W
        c.dmax2[:] = c.W
    return c


def hits_of(res, w):
    return [(int(h["i"]), int(h["j"]), h["score"].tobytes(), h["bias"].tobytes()) for h in res[res["win"] == w]]


def ref_hits(h):
    return [(i, j, np.float32(s).tobytes(), np.float32(b).tobytes()) for i, j, s, b in h]


CASES = [("small0", False), ("small2", True), ("trna", False), ("mb3", True)]


@pytest.mark.parametrize("name,nonbanded", CASES)
def test_calibrate_scan_matches_oracle(name, nonbanded):
    cm, g, _ = models(name)
    ccfg = cal.CalibrateConfig(nonbanded=nonbanded)
    lib_g, lib_l = cal.calibration_configs(cm, g.W, ccfg)
    L = 1500
    gen = cal.sample_genomic_sequences(7 + len(name), L, 3)
    frames = [gen[s * (L + 2):(s + 1) * (L + 2)] for s in range(3)]
    frames.append(frame(planted_seq(cm, 900, 0.45, 2, seed=5)))
    frames.append(frame(planted_seq(cm, 40, 0.5, 0, seed=6)))
    buf = np.concatenate(frames)
    offs = np.cumsum([0] + [len(f) for f in frames[:-1]])
    wins = np.array([(o, 1, len(f) - 2) for o, f in zip(offs, frames)], N.WINDOW_DTYPE)
    for local, libc in ((False, lib_g), (True, lib_l)):
        orc = oracle_calib_cfg(cm, local, g.W, ccfg.beta, nonbanded)
        sc = Scanner(libc)
        for inside in (False, True):
            for null3 in (True, False):
                res = cal.collect_scores(sc, inside, buf, wins, null3)
                for w, f in enumerate(frames):
                    ref = oracle.calib_scan(orc, int(inside), N.QDB2, f, 1, len(f) - 2, null3)
                    got = hits_of(res, w)
                    assert got == ref_hits(ref), (name, local, inside, null3, w, got[:3], ref[:3])
                    if len(f) > 1000:  # cutoff -inf keeps disjoint hits all along the window
                        assert len(got) >= (len(f) - 2) // (2 * libc.W), (len(got), libc.W)
        sc.close()


def test_calibrate_cm_matches_oracle_end_to_end():
    cm, g, _ = models("small2")
    ccfg = cal.CalibrateConfig(l_mb=0.005)
    n = cal.n_sequences(ccfg)
    assert n == 1
    res = cal.calibrate_cm(cm, ccfg, W=g.W)
    frames = oracle.genomic_sample(ccfg.seed, cal.EXPTAIL_CHUNKLEN, n)
    for mode in range(4):
        local, inside = cal.exp_mode_is_local(mode), cal.exp_mode_is_inside(mode)
        orc = oracle_calib_cfg(cm, local, g.W, ccfg.beta)
        scores = []
        for s in range(n):
            f = frames[s * (cal.EXPTAIL_CHUNKLEN + 2):(s + 1) * (cal.EXPTAIL_CHUNKLEN + 2)]
            scores += [h[2] for h in oracle.calib_scan(orc, int(inside), N.QDB2, f, 1, cal.EXPTAIL_CHUNKLEN, True)]
        ref = oracle.exp_fit(np.array(scores, np.float32), mode, n, cal.EXPTAIL_CHUNKLEN, 250, 750, 0.0,
                             float(n * cal.EXPTAIL_CHUNKLEN))
        got = res["exp"][mode]
        assert res["nhits"][mode] == len(scores) == got["nrandhits"] == ref["nrandhits"]
        for k in ("mu", "mu_orig", "tailp", "dbsize"):
            assert np.float64(got[k]).tobytes() == np.float64(ref[k]).tobytes(), (mode, k, got[k], ref[k])
        assert np.float64(got["lambda_"]).tobytes() == np.float64(ref["lambda"]).tobytes()
        assert got["lambda_"] > 0
    assert res["cells"] > 0 and res["kernel_ms"] > 0


def test_calibrate_rejects_sweep_kernel_and_small_L():
    cm, g, _ = models("small0")
    lib_g, _ = cal.calibration_configs(cm, g.W, cal.CalibrateConfig())
    sc = Scanner(lib_g)
    sc.set_kernel(N.KERNEL_SWEEP)
    f = frame(planted_seq(cm, 200, 0.5, 0, seed=1))
    with pytest.raises(N.CmgpuError, match="level kernel"):
        cal.collect_scores(sc, False, f, np.array([(0, 1, 200)], N.WINDOW_DTYPE), True)
    sc.close()
    with pytest.raises(N.CmgpuError):
        cal.calibrate_cm(cm, cal.CalibrateConfig(l_mb=0.001), W=g.W)
