"""CM files, no GPU: the reader takes the reference's own reader-test model
texts (src/cm_file.rs:2155-2212, v1.0 and v1.1) to the values those tests
assert; a model written in the INFERNAL1/a layout reads back with the same
state graph and probabilities within the file's 3-decimal log2 rounding, and
writing what was read is a fixed point; a read model configures to tables
equal to the oracle's independent restatement; the HMMER3/f filter block
reads back as the p7 profile, its composition and E-value parameters."""
import json
import os

import numpy as np
import pytest

import oracle
from infernox_b200 import cmfile, model, p7, synth

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "cm_file_kat.json")
STRUCT = ("sttype", "stid", "ndidx", "cfirst", "cnum", "plast", "pnum", "ndtype", "nodemap")


def test_reference_reader_tests():
    kat = json.load(open(GOLDEN))
    assert len(kat["models"]) == 2
    for m in kat["models"]:
        r = cmfile.read_cm(m["text"])
        assert (r.cm.name, r.cm.M, r.cm.st.nodes, r.cm.clen) == (m["name"], m["M"], m["nodes"], m["clen"])
        assert r.version == ("1.0" if m["text"].startswith("INFERNAL-1") else "1.1")
        # every distribution sums to one after the reader's renormalisation
        st = r.cm.st
        for v in range(r.cm.M):
            if st.cnum[v] > 0 and st.sttype[v] != synth.B_ST:
                assert abs(float(r.cm.t[v, :st.cnum[v]].sum()) - 1.0) < 1e-6
    v11 = cmfile.read_cm(kat["models"][1]["text"])
    assert v11.W == 10 and v11.acc == "RF00005" and v11.desc == "tRNA"
    # band columns in file order dmin2, dmin1, dmax1, dmax2 (src/cm_file.rs:637-644)
    assert [int(v11.bands[k][0]) for k in ("dmin2", "dmin1", "dmax1", "dmax2")] == [0, 5, 0, 10]
    # its ECMLC / ECMGC lines carry one value, not the six the reader needs: skipped
    assert v11.exp == {}


@pytest.mark.parametrize("seed,shape", [(5, "trna"), (9, (150, 0.4, 2, 3)), (12, (40, 0.3, 0, 1))])
def test_write_read_round_trip(seed, shape):
    ss = synth.trna_like() if shape == "trna" else synth.structure(*shape)
    cm = synth.synth_cm(ss, seed, name=f"rt{seed}")
    prof, _ = p7.synthetic_profile(cm.clen, seed)
    comp = p7.mean_composition(prof)
    ev = {"lmmu": -8.25, "lmlambda": 0.69, "lvmu": -9.5, "lvlambda": 0.69, "lftau": -5.75, "lflambda": 0.69}
    txt = cmfile.write_cm(cm, prof, comp, ev, max_length=300)
    r = cmfile.read_cm(txt)
    for k in STRUCT:
        assert np.array_equal(getattr(r.cm.st, k), getattr(cm.st, k)), k
    assert (r.cm.M, r.cm.clen, r.cm.st.nodes) == (cm.M, cm.clen, cm.st.nodes)
    # 3 decimals of log2 odds: relative error below 2^0.0005 - 1, then renormalised
    assert np.allclose(r.cm.t, cm.t, rtol=1e-3, atol=1e-7)
    assert np.allclose(r.cm.e, cm.e, rtol=1e-3, atol=1e-7)
    assert r.W == model.configure(cm, local=False).W
    # the filter block: 5 decimals of -ln p
    assert r.p7.M == prof.M and r.p7_max_length == 300 and r.p7_evparam == ev
    assert np.allclose(r.p7.mat, prof.mat, rtol=2e-5, atol=1e-7)
    assert np.allclose(r.p7.trans, prof.trans, rtol=2e-5, atol=1e-7)
    assert np.allclose(r.p7_compo, comp, rtol=2e-5)
    txt2 = cmfile.write_cm(r.cm, r.p7, r.p7_compo, r.p7_evparam, max_length=300)
    r2 = cmfile.read_cm(txt2)
    assert cmfile.write_cm(r2.cm, r2.p7, r2.p7_compo, r2.p7_evparam, max_length=300) == txt2
    # two models in one file
    both = cmfile.read_cms(txt + txt2)
    assert len(both) == 2 and both[1].cm.name == f"rt{seed}"


def test_read_model_configures_like_the_oracle():
    cm = synth.synth_cm(synth.structure(90, 0.4, 1, 4), 21, name="cfgtest")
    r = cmfile.read_cm(cmfile.write_cm(cm))
    for local in (False, True):
        mine = model.configure(r.cm, local=local)
        ref = oracle.prep_configure(r.cm, local)
        for k in ("tsc", "oesc", "itsc", "ioesc", "dmin1", "dmax1", "dmin2", "dmax2"):
            assert np.asarray(getattr(mine, k)).tobytes() == np.asarray(ref[k]).tobytes(), k
        assert mine.W == ref["W"]
    # the file's band columns are the band engine's on the model that was written
    g = model.configure(cm, local=False)
    for k in ("dmin1", "dmax1", "dmin2", "dmax2"):
        assert np.array_equal(r.bands[k], getattr(g, k))


def test_reader_rejects_non_cm_text():
    with pytest.raises(ValueError):
        cmfile.read_cm("HMMER3/f [3.1b2]\nNAME x\n//\n")
