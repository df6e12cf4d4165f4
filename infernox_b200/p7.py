"""P7 filter profiles and the GPU Viterbi filter.

Mirrors the reference's `build_vit_filter(&P7Profile) -> VitFilter` and
`vit_score(&VitFilter, dsq, l) -> Option<f32>` (src/p7_vitfilter.rs:121,
:292) over libcmscan_gpu.so; `vit_score_batch` scores many windows in one
launch.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _native as N


@dataclass
class P7Profile:
    """Match emissions mat[0..M][4] (row 0 unused) and transitions
    trans[0..M][7] = MM, MI, MD, IM, II, DM, DD (src/p7_hmm.rs:62-92)."""
    M: int
    mat: np.ndarray
    trans: np.ndarray


class VitFilter:
    def __init__(self, p: P7Profile, device: int = 0):
        self.p = p
        self._mat = np.ascontiguousarray(p.mat, np.float32).reshape(p.M + 1, 4)
        self._trans = np.ascontiguousarray(p.trans, np.float32).reshape(p.M + 1, 7)
        prof = N.P7Profile(p.M, N.ptr(self._mat, C.c_float), N.ptr(self._trans, C.c_float))
        self._h = C.c_void_p()
        N.check(N.lib().cmgpu_vit_filter_build(C.byref(prof), device, C.byref(self._h)))

    def close(self):
        if self._h:
            N.lib().cmgpu_vit_filter_free(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def tables(self):
        n = C.c_int32()
        sp = np.zeros(3, np.int16)
        N.lib().cmgpu_vit_filter_tables(self._h, None, 0, C.byref(n), None)
        tab = np.zeros(n.value, np.int16)
        N.check(N.lib().cmgpu_vit_filter_tables(self._h, tab.ctypes.data, n.value, C.byref(n), sp.ctypes.data))
        return tab, sp

    def score_batch(self, buf: np.ndarray, windows: np.ndarray):
        """Scores (f32 bits) and scored flags (0 = None, overflow) per window."""
        b = np.ascontiguousarray(buf, np.uint8)
        w = np.ascontiguousarray(windows, N.WINDOW_DTYPE)
        sc = np.zeros(len(w), np.float32)
        ok = np.zeros(len(w), np.uint8)
        N.check(N.lib().cmgpu_vit_score_batch(self._h, None, b.ctypes.data, b.size, w.ctypes.data, len(w),
                                              sc.ctypes.data, ok.ctypes.data))
        return sc, ok


def vit_score(f: VitFilter, dsq, l: int):
    """src/p7_vitfilter.rs:292 -- Some(score) or None."""
    a = np.ascontiguousarray(dsq, np.uint8)
    w = np.array([(0, 1, l)], N.WINDOW_DTYPE)
    sc, ok = f.score_batch(a, w)
    return float(sc[0]) if ok[0] else None
