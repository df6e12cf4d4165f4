"""A model read from a CM file runs the device path end to end: the CM
scanners (QDB1 CYK filter and QDB2 Inside) and the F1 -> F3b filter
cascade with the file's own HMMER3/f block (its composition and E-value
parameters) give the oracle's hits and windows bit for bit."""
import numpy as np
import pytest

import oracle
from infernox_b200 import _native as N
from infernox_b200 import cmfile, model, p7, scan, synth
from infernox_b200.scan import CYK_F32, INSIDE_I32, QDB1, QDB2

from helpers import frame, planted_seq

pytestmark = pytest.mark.gpu


def test_file_model_scans_and_filters_like_the_oracle():
    src = synth.synth_cm(synth.structure(110, 0.4, 2, 8), 33, name="filemodel")
    prof, cons = p7.synthetic_profile(src.clen, 33)
    ev = {"lmmu": -8.5, "lmlambda": 0.69, "lvmu": -9.0, "lvlambda": 0.69, "lftau": -6.0, "lflambda": 0.69}
    f = cmfile.read_cm(cmfile.write_cm(src, prof, p7.mean_composition(prof), ev, max_length=2 * src.clen))
    cm = f.cm
    n = 4000
    dsq = frame(planted_seq(cm, n, 0.5, 3, seed=5))
    loc = model.configure(cm, local=True)
    s = scan.Scanner(loc)
    for sr, band in ((CYK_F32, QDB1), (INSIDE_I32, QDB2)):
        ref, _, _, _ = oracle.qdb_scan(loc, sr, band, dsq, 1, n, 0.0, True)
        got = s.generic_scan(sr, band, dsq, 1, n, 0.0, True)
        assert len(ref) > 0
        assert [(h.i, h.j, np.float32(h.score).tobytes()) for h in got] == \
               [(h[0], h[1], np.float32(h[2]).tobytes()) for h in ref]
    # the filter cascade with the file's p7 block
    q = f.p7
    mf = p7.MsvFilter(q, f.p7_max_length, ev["lmmu"], ev["lmlambda"])
    ff = p7.FwdFilter(q, f.p7_compo, ev["lftau"], ev["lflambda"])
    cmw = loc.W
    got, acct = p7.f3_filter_batch(ff, dsq, np.array([(0, 1, n)], N.WINDOW_DTYPE), 0.35, 0.02, 0.02, cmw, mf=mf)
    want, wacct = oracle.f3_filter_sequence((q.M, q.mat, q.trans), f.p7_compo, ev["lftau"], ev["lflambda"], dsq,
                                            0.35, 0.02, 0.02, cmw, max_length=f.p7_max_length, mmu=ev["lmmu"],
                                            mlambda=ev["lmlambda"])
    assert [(int(r["start"]), int(r["end"]), np.float32(r["score"]).tobytes()) for r in got] == \
           [(a, b, np.float32(c).tobytes()) for a, b, c in want]
    assert acct == wacct and acct["n_past_msv"] > 0
