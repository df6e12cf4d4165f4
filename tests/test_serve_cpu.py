"""The serving loop's admission and queue logic on the host (no GPU): a
request larger than the budget and one sent to a full queue are refused
with their status, a cancelled request leaves the queue and is reported,
and admission takes requests in arrival order while the budget holds."""
import numpy as np

from infernox_b200 import serve

from helpers import models


def _server(budget=10_000, max_queue=3):
    cm, g, l = models("small0")
    return serve.Server([l], budget_residues=budget, max_queue=max_queue)


def _req(rid, n):
    return serve.Request(rid, np.zeros(n, np.uint8))


def test_refusals_and_cancel():
    s = _server()
    assert s.submit(_req(1, 6000)) == serve.REFUSED_TOO_LARGE  # 12000 residues > budget
    assert [s.submit(_req(k, 100)) for k in (2, 3, 4)] == [serve.OK] * 3
    r5 = _req(5, 100)
    assert s.submit(r5) == serve.REFUSED_QUEUE_FULL and r5.status == serve.REFUSED_QUEUE_FULL
    assert s.cancel(3) and not s.cancel(99)
    assert [r.rid for r in s.queue] == [2, 4]
    assert [r.rid for r in s.finished] == [3] and s.finished[0].status == serve.CANCELLED
    s.close()


def test_admission_in_order_within_budget():
    s = _server(budget=1000, max_queue=10)
    for k, n in enumerate((200, 250, 100, 30)):
        s.submit(_req(k, n))
    s._admit()  # 400 + 500 fit, the third (200) would pass 1000
    assert [r.rid for r in s.active] == [0, 1]
    assert [r.rid for r in s.queue] == [2, 3]
    assert all(r.remaining == 1 and r.start_model == 0 for r in s.active)
    s.close()


def test_envelopes_pad_and_merge():
    # hit (i, j) -> (j - (W-1), i + (W-1)) clipped to [1, n], merged where
    # they overlap, as cyk_seq_filter does
    assert serve._pad_merge([(10, 20), (15, 30), (200, 210)], 10, 300) == [(11, 19), (21, 24), (201, 209)]
    assert serve._pad_merge([(10, 20), (12, 22)], 10, 300) == [(11, 21)]
    assert serve._pad_merge([(1, 5)], 50, 30) == [(1, 30)]
    assert serve._pad_merge([], 10, 100) == []


def test_library_from_cm_file():
    """cmscan's CM database: a file of several models becomes the serving
    library, each model configured locally with the W its file states."""
    from infernox_b200 import cmfile, model, synth
    cms = [synth.synth_cm(synth.structure(c, 0.4, b, s), s, name=f"lib{s}") for c, b, s in
           ((40, 0, 1), (90, 1, 2), (60, 2, 3))]
    text = "".join(cmfile.write_cm(cm) for cm in cms)
    lib = serve.library_from_cm_file(text)
    assert [m.name for m in lib] == ["lib1", "lib2", "lib3"]
    assert all(m.local for m in lib)
    assert [m.W for m in lib] == [model.configure(cm, local=False).W for cm in cms]
    s = serve.Server(lib, budget_residues=10_000)
    assert s.submit(_req(1, 100)) == serve.OK
    s.close()
