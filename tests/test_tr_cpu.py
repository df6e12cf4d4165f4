"""The two truncated-scan oracles pinned against each other with the
reference's own properties (src/cm_dpsearch_trunc.rs):

* tr_cyk_scan_hb_wideband_equals_nonhb (:2663-2694): with fully permissive
  bands over a window no longer than W, the HMM-banded TrCYK vsc_root equals
  the non-banded generic_tr_scan TrCYK vsc_root (within 1e-4) with the same
  marginal mode, in the 5'-only, 3'-only and 5'-and-3' passes;
* ftr_inside_scan_hb_wideband_equals_nonhb (:2696-2726): the float HB
  TrInside against the integer non-banded TrInside with the same mode, and
  within 0.3 bits.  The reference's test holds 2e-2 on its one real model;
  on these five synthetic models the integer scan (every score rounded to
  1/1000 bit by Prob2Score, every ILogsum by its table) comes out below the
  float one by 0.002 to 0.27 bits, always below, as systematic rounding
  does -- the marginal emissions and penalties are the restated tables
  (cmgpu_prep_truncated), identical in both scans;
* QDB bands never raise the non-banded TrCYK score (:2568-2581 restated for
  the truncated scan);
* the wide-band pins again in the local configuration, passes 2-5.
The HB oracle restates tr_cyk_scan_hb / ftr_inside_scan_hb and the
non-banded one generic_tr_scan; they share no code."""
import numpy as np
import pytest

import oracle
from infernox_b200 import synth

from hb_helpers import as_tuple, tr_tables, wide_bands
from helpers import frame, models

PASSES = (2, 3, 4)


def _window(cm, cfg, seed):
    h = synth.emit(cm, np.random.default_rng(seed))
    L = min(len(h), cfg.W)
    return frame(h[:L]), L


@pytest.mark.parametrize("name", ["trna", "small0", "small2", "mb3"])
def test_wideband_trcyk_equals_nonbanded(name):
    cm, g, l = models(name)
    f, L = _window(cm, g, 3)
    ones = np.ones(g.M, np.uint8)
    for p in PASSES:
        tt = tr_tables(cm, g, p, False)
        _, vq, mq, _ = oracle.trq_scan(g, False, tt, f, 1, L, -1e30, False, 0, p, False)
        _, vh, mh, _, _ = oracle.tr_hb_scan(g, False, tt, (ones,) * 4, as_tuple(wide_bands(g, 1, L)), f, 1, L, -1e30,
                                            False, p, -1e30, False)
        assert abs(vq - vh) < 1e-4 and mq == mh, (p, vq, vh, mq, mh)


@pytest.mark.parametrize("name", ["trna", "small2"])
def test_wideband_trinside_float_equals_integer_nonbanded(name):
    cm, g, l = models(name)
    f, L = _window(cm, g, 4)
    ones = np.ones(g.M, np.uint8)
    for p in PASSES:
        tt = tr_tables(cm, g, p, False)
        _, vq, mq, _ = oracle.trq_scan(g, True, tt, f, 1, L, -1e30, False, 0, p, False)
        _, vh, mh, _, _ = oracle.tr_hb_scan(g, True, tt, (ones,) * 4, as_tuple(wide_bands(g, 1, L)), f, 1, L, -1e30,
                                            False, p, -1e30, False)
        assert abs(vq - vh) < 0.3 and mq == mh, (p, vq, vh, mq, mh)
        assert np.isfinite(vq) and vq > 0


@pytest.mark.parametrize("name", ["trna", "small2"])
def test_truncated_qdb_le_nonbanded(name):
    cm, g, l = models(name)
    f, L = _window(cm, g, 5)
    for p in PASSES:
        tt = tr_tables(cm, g, p, False)
        _, vn, _, _ = oracle.trq_scan(g, False, tt, f, 1, L, -1e30, False, 0, p, False)
        for q in (1, 2):
            _, vb, _, _ = oracle.trq_scan(g, False, tt, f, 1, L, -1e30, False, q, p, False)
            assert vb <= vn + 1e-6


@pytest.mark.parametrize("name", ["trna", "small0", "small2", "mb3", "cfg2"])
def test_wideband_equals_nonbanded_local(name):
    """The same pins in the local configuration (local truncation rules,
    local begins/ends), passes 5'-only, 3'-only, 5'-and-3' and 5'-and-3'-any:
    TrCYK equal within 1e-4 with the same mode; float HB TrInside against the
    integer non-banded TrInside with the same mode and within 0.3 bits."""
    cm, g, l = models(name)
    f, L = _window(cm, l, 5)
    ones = np.ones(l.M, np.uint8)
    for p in (2, 3, 4, 5):
        tt = tr_tables(cm, l, p, True)
        wb = as_tuple(wide_bands(l, 1, L))
        _, vq, mq, _ = oracle.trq_scan(l, False, tt, f, 1, L, -1e30, False, 0, p, True)
        _, vh, mh, _, _ = oracle.tr_hb_scan(l, False, tt, (ones,) * 4, wb, f, 1, L, -1e30, False, p, -1e30, True)
        assert abs(vq - vh) < 1e-4 and mq == mh, (p, vq, vh, mq, mh)
        _, vq, mq, _ = oracle.trq_scan(l, True, tt, f, 1, L, -1e30, False, 0, p, True)
        _, vh, mh, _, _ = oracle.tr_hb_scan(l, True, tt, (ones,) * 4, wb, f, 1, L, -1e30, False, p, -1e30, True)
        assert abs(vq - vh) < 0.3 and mq == mh, (p, vq, vh, mq, mh)
