"""MSV filter tables and the SSV trigger threshold built by the library's host
code (build_msv_filter, src/cm_pipeline.rs:201-340; ssv_diagonals' sc_thresh,
:522-533) against the oracle's restatement.  No GPU: filters are built with
device = -1."""
import numpy as np
import pytest

import oracle
from infernox_b200 import _native as N
from infernox_b200.p7 import MsvFilter

from p7_helpers import MS, Lcg, peaked_profile, random_profile


def profiles():
    rng = Lcg()
    out = [random_profile(rng, m) for m in MS]
    out += [peaked_profile(7 + m, m)[0] for m in (350, 1000, 2048)]
    return out


@pytest.mark.parametrize("max_length", [1, 90, 1900])
def test_msv_tables_match_oracle(max_length):
    for p in profiles():
        f = MsvFilter(p, max_length, device=-1)
        rbv, b5, pre, suf, sc = f.tables()
        orbv, ob5, opre, osuf, osc = oracle.msv_tables(p.M, p.mat, p.trans, max_length)
        assert np.array_equal(rbv, orbv), p.M
        assert np.array_equal(b5, ob5), p.M
        assert np.array_equal(pre.view(np.uint32), opre.view(np.uint32)), p.M
        assert np.array_equal(suf.view(np.uint32), osuf.view(np.uint32)), p.M
        assert sc.tobytes() == np.float32(osc).tobytes()
        f.close()


@pytest.mark.parametrize("f1", [1e-10, 0.02, 0.35, 0.9])
@pytest.mark.parametrize("mmu,mlambda", [(-8.0, 0.69), (-11.5, 0.72), (2.0, 0.6)])
def test_ssv_threshold_matches_oracle(f1, mmu, mlambda):
    for p in profiles()[::4]:
        f = MsvFilter(p, 150, mmu, mlambda, device=-1)
        assert f.threshold(f1) == oracle.ssv_threshold(p.M, p.mat, p.trans, 150, mmu, mlambda, f1)
        f.close()


def test_msv_rejects_models_over_2048_positions():
    p, _ = peaked_profile(3, 2049)
    with pytest.raises(N.CmgpuError) as e:
        MsvFilter(p, 100, device=-1)
    assert e.value.rc == -7
