"""The allocation-free window scan (cmgpu_qdb_scan_noalloc) against the
regular one (cmgpu_qdb_scan), through the C ABI.

The no-allocation entry point serves callers that cannot call cudaMalloc or
cudaFree while they scan: processes whose device memory belongs to a
framework's caching allocator or a fixed budget, and processes running other
streams that cannot accept the device-wide synchronisation of cudaFree.  It
keeps its scratch in a fixed 16 MiB device array shared by every call on a
GPU.  Its hits must equal the regular entry point's exactly, and two calls in
a row must not see each other's leftovers.  This file is collected last so
that a run stopping at the first failure has run every other test first.
"""
import ctypes as C

import numpy as np
import pytest

from infernox_b200 import _native as N
from infernox_b200.scan import CYK_F32, INSIDE_I32, KERNEL_LEVEL, NOQDB, QDB1, QDB2, Scanner

from helpers import frame, models, planted_seq

pytestmark = pytest.mark.gpu


def noalloc_scan(sc: Scanner, semiring, band, dsq, i0, j0, cutoff, null3):
    cap = 4096
    out = np.zeros(cap, N.HIT_DTYPE)
    nout = C.c_int32()
    rc = N.lib().cmgpu_qdb_scan_noalloc(sc._model, None, semiring, band, N.ptr(dsq, C.c_uint8),
                                        len(dsq) - 2, i0, j0, float(cutoff), int(null3),
                                        out.ctypes.data, cap, C.byref(nout))
    N.check(rc)
    return [(int(h["i"]), int(h["j"]), h["score"].tobytes(), h["bias"].tobytes()) for h in out[: nout.value]]


def regular_scan(sc: Scanner, semiring, band, dsq, i0, j0, cutoff, null3):
    return [(h.i, h.j, np.float32(h.score).tobytes(), np.float32(h.bias).tobytes())
            for h in sc.generic_scan(semiring, band, dsq, i0, j0, cutoff, null3)]


def test_noalloc_matches_regular_scan_two_calls_in_a_row():
    cm, g, l = models("trna")
    sc = Scanner(l)
    a = frame(planted_seq(cm, 5000, 0.5, 4, seed=901))
    b = frame(planted_seq(cm, 3000, 0.45, 3, seed=902))
    # first call: integer Inside, QDB2 (decks in shared memory)
    got1 = noalloc_scan(sc, INSIDE_I32, QDB2, a, 1, 5000, 0.0, True)
    # second call right after: CYK QDB1 on another sequence and window
    got2 = noalloc_scan(sc, CYK_F32, QDB1, b, 101, 2900, 0.0, True)
    assert got1 == regular_scan(sc, INSIDE_I32, QDB2, a, 1, 5000, 0.0, True) and got1
    assert got2 == regular_scan(sc, CYK_F32, QDB1, b, 101, 2900, 0.0, True) and got2


def one_lane_fits_in_smem(cfg, semiring, band) -> bool:
    """Whether one work item's decks fit in shared memory: the criterion both
    the regular path (level kernel, one lane forced) and the no-allocation
    path use."""
    sc = Scanner(cfg)
    try:
        sc.set_kernel(KERNEL_LEVEL)
        sc.set_shape(1, 512, 0, 1)
        dsq = np.concatenate([[255], np.zeros(300, np.uint8), [255]]).astype(np.uint8)
        sc.generic_scan(semiring, band, dsq, 1, 300, 1e9, False)
        return bool(sc.stats()["deck_in_smem"])
    finally:
        sc.close()


def test_noalloc_global_decks_two_calls_in_a_row():
    """A model whose non-banded decks do not fit in shared memory: the decks
    live in the static array; the second call must not see the first's."""
    cm, g, l = models("cfg2")
    assert not one_lane_fits_in_smem(l, INSIDE_I32, NOQDB), "this case must take the global-deck branch"
    sc = Scanner(l)
    a = frame(planted_seq(cm, 1500, 0.45, 2, seed=903))
    for _ in range(2):
        got = noalloc_scan(sc, INSIDE_I32, NOQDB, a, 1, 1500, 0.0, True)
        assert got == regular_scan(sc, INSIDE_I32, NOQDB, a, 1, 1500, 0.0, True) and got


def test_noalloc_rejects_oversized_request():
    cm, g, l = models("small0")
    sc = Scanner(l)
    big = np.zeros(20_000_002, np.uint8)   # 20 M residues: more than the 16 MiB array holds
    big[0] = big[-1] = 255
    out = np.zeros(16, N.HIT_DTYPE)
    nout = C.c_int32()
    rc = N.lib().cmgpu_qdb_scan_noalloc(sc._model, None, CYK_F32, QDB1, N.ptr(big, C.c_uint8),
                                        len(big) - 2, 1, len(big) - 2, 0.0, 0, out.ctypes.data, 16,
                                        C.byref(nout))
    assert rc == -7  # CMGPU_ENOSPACE
    assert b"16 MiB" in N.lib().cmgpu_last_error()
