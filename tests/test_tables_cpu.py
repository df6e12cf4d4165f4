"""The library's model preparation against the oracle's independent
restatement of the same reference builders (oracle/prep_oracle.c), bit for
bit, on every test model shape, global and local configuration -- no GPU.

Score tables and bands (cmgpu_prep_configure): cm_config_local,
cm_logoddsify, build_integer_scores, the QDB band engine and W.
Truncated-scan inputs (cmgpu_prep_truncated): fill_marginal_emissions,
TrPenalties::new (from the expected state occupancy and the emit map) and
the node spans allow_truncation reads.

Every parity test compares the GPU with the oracle scanning the library's
tables; this file closes the loop: those tables equal the oracle's own."""
import numpy as np
import pytest

import oracle
from infernox_b200 import hb

from helpers import models

NAMES = ["cfg0", "small0", "small2", "mb3", "cfg2", "cfg3"]
CONFIG_FIELDS = ["tsc", "oesc", "endsc", "beginsc", "itsc", "ioesc", "iendsc", "ibeginsc",
                 "dmin1", "dmax1", "dmin2", "dmax2", "t_local"]


def same_bits(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return a.shape == b.shape and a.tobytes() == b.tobytes()


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("local", [False, True], ids=["global", "local"])
def test_score_tables_and_bands_match_oracle(name, local):
    cm, g, l = models(name)
    mine = l if local else g
    ref = oracle.prep_configure(cm, local)
    bad = [k for k in CONFIG_FIELDS if not same_bits(getattr(mine, k), ref[k])]
    assert not bad, bad
    assert (mine.W, mine.flags, mine.iel_selfsc) == (ref["W"], ref["flags"], ref["iel_selfsc"])
    assert np.float32(mine.el_selfsc).tobytes() == np.float32(ref["el_selfsc"]).tobytes()


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("local", [False, True], ids=["global", "local"])
def test_truncated_inputs_match_oracle(name, local):
    cm, g, l = models(name)
    mine = hb.truncated_tables(cm, local)
    ref = oracle.prep_truncated(cm, local)
    bad = [k for k in ref if not same_bits(mine[k], ref[k])]
    assert not bad, bad


def test_truncated_penalties_are_probabilities_in_log_space():
    """Properties the reference's construction implies: every qualifying
    state's local penalty is finite and negative (a log2 probability), the
    global 5'-and-3' row is set wherever the local one is, and ROOT_S itself
    is never a truncated entry."""
    cm, g, l = models("cfg2")
    loc, glb = oracle.prep_truncated(cm, True), oracle.prep_truncated(cm, False)
    fin = loc["pty"][0] > -1e30
    assert fin.sum() > cm.M // 3
    assert (loc["pty"][:, fin] < 0).all()
    assert (glb["pty"][0][fin] > -1e30).all()
    assert loc["pty"][0][0] < -1e30 and glb["pty"][0][0] < -1e30


@pytest.mark.parametrize("name", ["cfg0", "small2", "mb3", "cfg2"])
def test_calibration_configurations_match_oracle(name):
    """cmcalibrate's two configurations (both band sets at beta 1e-15 on the
    global transitions, the model's W kept) against the oracle's builders."""
    from infernox_b200 import calibrate as cal
    cm, g, l = models(name)
    ccfg = cal.CalibrateConfig()
    for local, mine in zip((False, True), cal.calibration_configs(cm, g.W, ccfg)):
        ref = oracle.prep_configure(cm, local, g.W, ccfg.beta, ccfg.beta)
        bad = [k for k in CONFIG_FIELDS if not same_bits(getattr(mine, k), ref[k])]
        assert not bad, bad
        assert mine.W == ref["W"] == g.W
        # the tighter beta widens every band
        assert (mine.dmax2 >= g.dmax2).all() and (mine.dmin2 <= g.dmin2).all()
