"""The oracle pinned against the reference's own known-answer tests and
properties (fixtures in tests/golden/, extracted from the reference's test
modules by tests/golden/make_golden.py)."""
import json
import os

import numpy as np
import pytest

import oracle
from infernox_b200 import _native as N
from infernox_b200.scan import CYK_F32, INSIDE_I32, NOQDB, QDB1, QDB2

from helpers import frame, models, planted_seq

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    with open(os.path.join(GOLD, name)) as f:
        return json.load(f)


def test_ilogsum_table_kats():
    """src/cp9.rs:91-101 table entries and :104-116 endpoints."""
    g = load("ilogsum_kat.json")
    t = oracle.ilogsum_table()
    for i, v in g["table"]:
        assert t[i] == v, (i, t[i], v)
    assert t[0] == 1000 and t[22999] == 0
    # the product's table (uploaded to the device) is the same table
    import ctypes as C
    p = np.zeros(23000, np.int32)
    N.lib().cmgpu_ilogsum_table(p.ctypes.data_as(C.POINTER(C.c_int32)), 23000)
    assert np.array_equal(p, t)
    assert np.all(np.diff(t) <= 0) and np.all(np.diff(t) >= -1)


def test_ilogsum_edge_kats():
    """src/cp9.rs:81-88 sentinel and bound cases, :110 ilogsum(500,500)."""
    g = load("ilogsum_kat.json")
    for a, b, want in g["calls"]:
        assert oracle.ilogsum(a, b) == want, (a, b)


def test_state_delta_kats():
    """src/cm_qdband.rs:639-690."""
    g = load("state_delta_kat.json")
    from infernox_b200 import synth
    delta = {synth.D_ST: 0, synth.MP_ST: 2, synth.ML_ST: 1, synth.MR_ST: 1, synth.IL_ST: 1,
             synth.IR_ST: 1, synth.S_ST: 0, synth.E_ST: 0, synth.B_ST: 0, synth.EL_ST: 0}
    for st, d in g["state_delta"]:
        assert delta[st] == d


@pytest.mark.parametrize("name", ["trna", "small2"])
def test_qdb_scan_never_exceeds_nonbanded(name):
    """Bands only remove parses: best QDB score <= best non-banded score
    (the property of src/cm_dpsearch_trunc.rs:2568-2581, standard scanner)."""
    cm, g, l = models(name)
    n = 600
    dsq = frame(planted_seq(cm, n, 0.5, 1, seed=31))
    for sr, band in ((CYK_F32, QDB1), (INSIDE_I32, QDB2)):
        hb, cb, _, _ = oracle.qdb_scan(l, sr, band, dsq, 1, n, -1e9, False, want_cands=True)
        hn, cn, _, _ = oracle.qdb_scan(l, sr, NOQDB, dsq, 1, n, -1e9, False, want_cands=True)
        best_b = {(j, d): s for j, d, s in cb}
        best_n = {(j, d): s for j, d, s in cn}
        for k, s in best_b.items():
            assert s <= best_n[k] + 1e-6


def test_inside_at_least_cyk():
    """Inside sums the parses CYK maximises (cf. src/cm_dpsearch_trunc.rs:2587):
    per cell, Inside >= CYK up to the 1/1000-bit integer rounding."""
    cm, g, l = models("trna")
    n = 500
    dsq = frame(planted_seq(cm, n, 0.5, 1, seed=32))
    _, cc, _, _ = oracle.qdb_scan(l, CYK_F32, NOQDB, dsq, 1, n, -1e9, False, want_cands=True)
    _, ci, _, _ = oracle.qdb_scan(l, INSIDE_I32, NOQDB, dsq, 1, n, -1e9, False, want_cands=True)
    ins = {(j, d): s for j, d, s in ci}
    checked = 0
    for j, d, s in cc:
        if (j, d) in ins and s > -1e5:
            assert ins[(j, d)] >= s - 0.001 * (2 * d + 10), (j, d)
            checked += 1
    assert checked > 1000


def test_planted_homolog_found():
    cm, g, l = models("trna")
    n = 3000
    rng = np.random.default_rng(1)
    from infernox_b200 import synth
    seq = synth.random_dsq(n, 0.5, rng)
    h = synth.emit(cm, rng)
    seq[1000:1000 + len(h)] = h
    hits, _, _, _ = oracle.qdb_scan(l, CYK_F32, QDB1, frame(seq), 1, n, 10.0, True)
    assert any(abs(i - 1001) < 10 and abs(j - (1000 + len(h))) < 10 for i, j, _, _ in hits)


def test_counts_equal_product_counter():
    cm, g, l = models("mb3")
    n = 400
    dsq = frame(planted_seq(cm, n, 0.5, 0, seed=2))
    for sr, band in ((CYK_F32, QDB1), (INSIDE_I32, QDB2), (INSIDE_I32, NOQDB)):
        _, _, cells, terms = oracle.qdb_scan(l, sr, band, dsq, 1, n, 0.0, False)
        assert l.count_work(sr, band, n) == (cells, terms)


def test_regression_fixture():
    """Oracle output on a fixed model and sequence (tests/golden/scan_small.json)."""
    g = load("scan_small.json")
    cm, gl, l = models(g["model"])
    c = l if g["local"] else gl
    dsq = frame(planted_seq(cm, g["n"], 0.5, g["nplant"], seed=g["seed"]))
    for case in g["cases"]:
        hits, _, _, _ = oracle.qdb_scan(c, case["semiring"], case["band"], dsq, 1, g["n"],
                                        case["cutoff"], True)
        assert [[h[0], h[1], round(h[2], 4), round(h[3], 6)] for h in hits] == case["hits"]
