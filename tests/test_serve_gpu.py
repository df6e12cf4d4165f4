"""The serving loop on the GPU: every request's hits are the same when it is
scanned alone (model by model through cyk_seq_filter and final_stage_inside,
the reference's per-query loop) and when it shares batches with other
requests -- including requests that join while the library cursor is
mid-way round -- and the same again on a server that holds only that
request.  Exact equality of every hit (i, j, score, bias)."""
import numpy as np
import pytest

from infernox_b200 import serve, synth

from helpers import models, planted_seq

pytestmark = pytest.mark.gpu


def _requests(lib_cms, n, seed):
    rng = np.random.default_rng(seed)
    reqs = []
    for k in range(n):
        L = int(np.exp(rng.uniform(np.log(150), np.log(2500))))
        src = lib_cms[int(rng.integers(len(lib_cms)))]
        seq = planted_seq(src, L, float(rng.uniform(0.4, 0.6)), 1 if rng.random() < 0.6 else 0,
                          seed=int(rng.integers(1 << 30)))
        reqs.append(serve.Request(k, seq))
    return reqs


def test_request_hits_alone_equal_mixed():
    names = ("small0", "small2", "cfg0", "mb3")
    cms = [models(n)[0] for n in names]
    lib = [models(n)[2] for n in names]
    reqs = _requests(cms, 7, 11)
    srv = serve.Server(lib, budget_residues=12_000, f6_cutoff=0.0, final_cutoff=5.0)
    for r in reqs[:3]:
        assert srv.submit(r) == serve.OK
    srv.step()
    srv.step()  # the cursor is mid-way round when the rest arrive
    for r in reqs[3:]:
        assert srv.submit(r) == serve.OK
    steps = 0
    while not srv.idle():
        srv.step()
        steps += 1
        assert steps < 200
    assert sorted(r.rid for r in srv.finished) == list(range(7))
    assert any(r.start_model != 0 for r in srv.finished)  # some joined mid-way round
    nhits = 0
    for r in reqs:
        alone = serve.scan_alone(srv, r)
        assert set(r.hits) == set(alone)
        for key in alone:
            assert r.hits[key] == alone[key], (r.rid, key)
            nhits += len(alone[key])
    assert nhits > 0
    # one request on a server of its own
    solo = serve.Server(lib, budget_residues=12_000, f6_cutoff=0.0, final_cutoff=5.0)
    r = serve.Request(99, reqs[4].seq)
    solo.submit(r)
    while not solo.idle():
        solo.step()
    assert r.hits == reqs[4].hits
    srv.close()
    solo.close()


def test_budget_limits_active_residues():
    cms = [models("small0")[0]]
    lib = [models("small0")[2]]
    reqs = _requests(cms, 6, 12)
    budget = 2 * max(len(r.seq) for r in reqs) + 10
    srv = serve.Server(lib, budget_residues=budget)
    for r in reqs:
        srv.submit(r)
    while not srv.idle():
        srv._admit()
        assert sum(r.residues for r in srv.active) <= budget
        srv.step()
    assert len(srv.finished) == 6
    srv.close()
