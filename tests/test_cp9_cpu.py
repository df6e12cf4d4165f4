"""The CP9 HMM of a CM, no GPU: the library's builder (cmgpu_prep_cp9,
cp9_build_and_configure, src/cp9.rs:2212-2232) equals the oracle's
independent restatement bit for bit -- probabilities, integer scores and the
HMM -> CM state map -- on every test model shape; the transition index both
take for a parent / child pair is the reference's transition map's
(tests/golden/tmap_kat.json, src/cp9.rs:480-740); and the HMM is a
probability model in local mode."""
import json
import os

import numpy as np
import pytest

import oracle
from infernox_b200 import model, synth

from helpers import models

NAMES = ["trna", "small0", "small2", "cfg2", "mb3", "cfg3"]


@pytest.mark.parametrize("name", NAMES)
def test_cp9_matches_oracle(name):
    cm, _, _ = models(name)
    mine, ref = model.cp9(cm), oracle.prep_cp9(cm)
    bad = [k for k in mine if np.asarray(mine[k]).tobytes() != np.asarray(ref[k]).tobytes()]
    assert not bad, bad


def test_transition_index_is_the_reference_map():
    """Every parent / child pair the occupancy and subpath sums visit: the
    reference looks the transition up in its map under (parent's unique
    state, node type of the child -- the next node's for an insert --,
    child's unique state); the child's offset among the parent's children
    (0 for a bifurcation's children) is that entry."""
    kat = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "tmap_kat.json")))
    tmap = {(a, b, c): n for a, b, c, n in kat["entries"]}
    assert len(tmap) == len(kat["entries"]) == 264
    checked = 0
    for name in NAMES:
        cm, _, _ = models(name)
        st = cm.st
        for v in range(cm.M):
            ins = 1 if st.sttype[v] in (synth.IL_ST, synth.IR_ST) else 0
            for y in range(st.pnum[v] - 1, ins - 1, -1):
                x = st.plast[v] - y
                key = (int(st.stid[x]), int(st.ndtype[st.ndidx[v] + ins]), int(st.stid[v]))
                want = 0 if st.sttype[x] == synth.B_ST else v - st.cfirst[x]
                assert tmap.get(key) == want, (name, x, v, key)
                checked += 1
    assert checked > 10000


@pytest.mark.parametrize("name", ["trna", "cfg2", "cfg3"])
def test_cp9_is_a_local_probability_model(name):
    cm, _, _ = models(name)
    h = model.cp9(cm)
    H = cm.clen
    t = h["t"].astype(np.float64)
    assert abs(h["begin"][1:].sum() + t[0, 1] + t[0, 2] + t[0, 3] - 1.0) < 1e-5
    assert np.allclose(t[1:, 0:4].sum(1) + h["end"][1:], 1.0, atol=1e-5)  # out of M_k: MM MI MD MEL + end
    assert np.allclose(t[:, 4:7].sum(1), 1.0, atol=1e-5)                   # out of I_k
    assert np.allclose(t[1:, 7:10].sum(1), 1.0, atol=1e-5)                 # out of D_k
    assert np.allclose(h["mat"][1:].sum(1), 1.0, atol=1e-5) and np.allclose(h["ins"].sum(1), 1.0, atol=1e-5)
    # local mode: every position can be entered and left; end-local exits where nodes have them
    assert (h["begin"][1:] > 0).all() and (h["end"][1:] > 0).all()
    el = h["has_el"][1:] == 1  # node 0's flag (a bifurcation at the first column) takes no exit
    assert el.sum() > 0 and (t[1:][el, 3] > 0).all() and (t[1:][~el, 3] == 0).all()
    # the exits' sources are the flagged nodes; each exit lands to the right of its source
    pairs = h["el_pairs"]
    assert set(pairs[:, 0].tolist()) == set(np.nonzero(h["has_el"])[0].tolist())
    assert (pairs[:, 1] > pairs[:, 0]).all() and (pairs[:, 1] <= H + 1).all()
    # every HMM node's match and insert states come from the CM
    assert (h["hns2cs"][:, 0, 0] >= 0).all() and (h["hns2cs"][:, 1, 0] >= 0).all()
    assert (h["hns2cs"][1:, 2, 0] >= 0).all()
    # the integer scores are the probabilities' log-odds
    assert h["otsc"][1, 0] == int(np.floor(0.5 + 1000 * np.log(np.float32(t[1, 0])) * 1.44269504))


def test_cp9_rejects_a_wrong_length():
    cm, _, _ = models("small0")
    import ctypes as C
    from infernox_b200 import _native as N
    p, keep = model.params_struct(cm)
    s = N.Cp9()
    s.M = cm.clen + 1
    with pytest.raises(N.CmgpuError):
        N.check(N.lib().cmgpu_prep_cp9(C.byref(p), C.byref(s)))
