"""The HMM-banded oracle pinned against the QDB oracle and the reference's
band properties, on CPU.

* Wide bands give the non-banded answer: with fully permissive bands over
  an envelope no longer than W, the HB CYK vsc_root equals the largest ROOT
  cell of the non-banded QDB scan (the standard-CM analogue of the
  reference's wide-band test, src/cm_dpsearch_trunc.rs:2617-2726).
* Narrower bands never raise the CYK score (a subset of parses).
* Inside >= CYK on the same bands (src/cm_dpsearch_trunc.rs:2587).
"""
import numpy as np
import pytest

import oracle

from hb_helpers import as_tuple, qdb_bands, ragged_bands, wide_bands
from helpers import frame, models, planted_seq


@pytest.mark.parametrize("name", ["trna", "small2", "mb3"])
@pytest.mark.parametrize("loc", [False, True])
def test_hb_oracle_wide_bands_equal_nonbanded(name, loc):
    cm, g, l = models(name)
    cfg = l if loc else g
    seq = frame(planted_seq(cm, 300, 0.5, 2, seed=77))
    for i0 in (1, 120):
        j0 = min(i0 + cfg.W - 1, 300)
        v, _, _, _ = oracle.hb_scan(cfg, False, as_tuple(wide_bands(cfg, i0, j0)), seq, i0, j0, 0.0, False, 0.0, False)
        _, cands, _, _ = oracle.qdb_scan(cfg, 0, 0, seq, i0, j0, -1e30, False, want_cands=True)
        best = max(c[2] for c in cands)
        assert abs(v - best) <= 1e-4 * max(1.0, abs(best)), (v, best)


@pytest.mark.parametrize("name", ["trna", "small2"])
def test_hb_oracle_band_monotone_and_inside_ge_cyk(name):
    cm, g, l = models(name)
    seq = frame(planted_seq(cm, 300, 0.5, 2, seed=78))
    i0, j0 = 30, 30 + l.W - 1
    vw = oracle.hb_scan(l, False, as_tuple(wide_bands(l, i0, j0)), seq, i0, j0, 0.0, False, 0.0, False)[0]
    for b in (qdb_bands(l, i0, j0), ragged_bands(l, i0, j0, 4)):
        vc = oracle.hb_scan(l, False, as_tuple(b), seq, i0, j0, 0.0, False, 0.0, False)[0]
        vi = oracle.hb_scan(l, True, as_tuple(b), seq, i0, j0, 0.0, False, 0.0, False)[0]
        assert vc <= vw + 1e-6
        assert vi >= vc - 1e-2
