"""Configured covariance models: the scanner's view of a CM.

``configure(cm, local=True)`` runs the library's host-side model preparation
(cmgpu_prep_configure) on a probability-level model, producing the score
tables and query-dependent bands exactly as the reference's searcher builds
them for the --nohmm / --max scan paths (src/cm_search.rs:899-979):

* local=False: the global CM (`cm_global`: global scores, QDB bands, W);
* local=True:  the local scan CM (`cm_local_scan`: localised begins/ends,
  integer scores, bands copied from the global model).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _native as N
from .synth import SynthCM

DEFAULT_BETA_W = 1e-7
DEFAULT_BETA_QDB1 = 1e-7
DEFAULT_BETA_QDB2 = 1e-15


@dataclass
class ConfiguredCM:
    """Score tables + bands of one configured CM (numpy arrays own the data)."""
    name: str
    M: int
    W: int
    flags: int
    clen: int
    sttype: np.ndarray
    stid: np.ndarray
    cfirst: np.ndarray
    cnum: np.ndarray
    tsc: np.ndarray      # [M,6] f32
    oesc: np.ndarray     # [M,324] f32
    endsc: np.ndarray
    beginsc: np.ndarray
    el_selfsc: float
    itsc: np.ndarray     # [M,6] i32
    ioesc: np.ndarray    # [M,324] i32
    iendsc: np.ndarray
    ibeginsc: np.ndarray
    iel_selfsc: int
    dmin1: np.ndarray
    dmax1: np.ndarray
    dmin2: np.ndarray
    dmax2: np.ndarray
    null: np.ndarray
    n3_omega: float
    t_local: np.ndarray
    _struct: N.Cm = None

    @property
    def local(self) -> bool:
        return bool(self.flags & (1 << 10))

    def as_struct(self) -> N.Cm:
        """cmgpu_cm view; the arrays stay owned by this object."""
        if self._struct is None:
            s = N.Cm()
            s.M, s.W, s.flags = self.M, self.W, self.flags
            s.sttype = N.ptr(self.sttype, C.c_int8)
            s.stid = N.ptr(self.stid, C.c_int8)
            s.cfirst = N.ptr(self.cfirst, C.c_int32)
            s.cnum = N.ptr(self.cnum, C.c_int32)
            s.tsc = N.ptr(self.tsc, C.c_float)
            s.oesc = N.ptr(self.oesc, C.c_float)
            s.endsc = N.ptr(self.endsc, C.c_float)
            s.beginsc = N.ptr(self.beginsc, C.c_float)
            s.el_selfsc = self.el_selfsc
            s.itsc = N.ptr(self.itsc, C.c_int32)
            s.ioesc = N.ptr(self.ioesc, C.c_int32)
            s.iendsc = N.ptr(self.iendsc, C.c_int32)
            s.ibeginsc = N.ptr(self.ibeginsc, C.c_int32)
            s.iel_selfsc = self.iel_selfsc
            s.dmin1 = N.ptr(self.dmin1, C.c_int32)
            s.dmax1 = N.ptr(self.dmax1, C.c_int32)
            s.dmin2 = N.ptr(self.dmin2, C.c_int32)
            s.dmax2 = N.ptr(self.dmax2, C.c_int32)
            for a in range(4):
                s.null[a] = float(self.null[a])
            s.n3_omega = self.n3_omega
            self._struct = s
        return self._struct

    def count_work(self, semiring: int, qdbidx: int, L: int):
        """Exact (cells, terms) the reference scanner evaluates on a window of length L."""
        c, t = C.c_double(), C.c_double()
        N.check(N.lib().cmgpu_count_work(C.byref(self.as_struct()), semiring, qdbidx, int(L),
                                         C.byref(c), C.byref(t)))
        return c.value, t.value


def params_struct(cm: SynthCM):
    st = cm.st
    keep = dict(
        sttype=np.ascontiguousarray(st.sttype, np.int8), stid=np.ascontiguousarray(st.stid, np.int8),
        ndtype=np.ascontiguousarray(st.ndtype, np.int8), ndidx=np.ascontiguousarray(st.ndidx, np.int32),
        cfirst=np.ascontiguousarray(st.cfirst, np.int32), cnum=np.ascontiguousarray(st.cnum, np.int32),
        plast=np.ascontiguousarray(st.plast, np.int32), pnum=np.ascontiguousarray(st.pnum, np.int32),
        nodemap=np.ascontiguousarray(st.nodemap, np.int32),
        t=np.ascontiguousarray(cm.t, np.float32), e=np.ascontiguousarray(cm.e, np.float32),
    )
    p = N.CmParams()
    p.M, p.nodes, p.clen = st.M, st.nodes, st.clen
    p.sttype = N.ptr(keep["sttype"], C.c_int8)
    p.stid = N.ptr(keep["stid"], C.c_int8)
    p.ndtype = N.ptr(keep["ndtype"], C.c_int8)
    p.ndidx = N.ptr(keep["ndidx"], C.c_int32)
    p.cfirst = N.ptr(keep["cfirst"], C.c_int32)
    p.cnum = N.ptr(keep["cnum"], C.c_int32)
    p.plast = N.ptr(keep["plast"], C.c_int32)
    p.pnum = N.ptr(keep["pnum"], C.c_int32)
    p.nodemap = N.ptr(keep["nodemap"], C.c_int32)
    p.t = N.ptr(keep["t"], C.c_float)
    p.e = N.ptr(keep["e"], C.c_float)
    for a in range(4):
        p.null[a] = float(cm.null[a])
    p.el_selfsc = cm.el_selfsc
    p.pbegin = cm.pbegin
    p.pend = cm.pend
    p.n3_omega = cm.n3_omega
    return p, keep


def configure(cm: SynthCM, local: bool = True, W: int = 0, beta1: float = DEFAULT_BETA_QDB1,
              beta2: float = DEFAULT_BETA_QDB2, betaW: float = DEFAULT_BETA_W) -> ConfiguredCM:
    M = cm.M
    p, keep = params_struct(cm)
    out = dict(
        tsc=np.zeros((M, 6), np.float32), oesc=np.zeros((M, 324), np.float32),
        endsc=np.zeros(M, np.float32), beginsc=np.zeros(M, np.float32),
        itsc=np.zeros((M, 6), np.int32), ioesc=np.zeros((M, 324), np.int32),
        iendsc=np.zeros(M, np.int32), ibeginsc=np.zeros(M, np.int32),
        dmin1=np.zeros(M, np.int32), dmax1=np.zeros(M, np.int32),
        dmin2=np.zeros(M, np.int32), dmax2=np.zeros(M, np.int32),
        t_local=np.zeros((M, 6), np.float32),
    )
    s = N.CmScores()
    for k in ("tsc", "oesc", "endsc", "beginsc", "t_local"):
        setattr(s, k, N.ptr(out[k], C.c_float))
    for k in ("itsc", "ioesc", "iendsc", "ibeginsc", "dmin1", "dmax1", "dmin2", "dmax2"):
        setattr(s, k, N.ptr(out[k], C.c_int32))
    N.check(N.lib().cmgpu_prep_configure(C.byref(p), int(local), int(W), beta1, beta2, betaW,
                                         C.byref(s)))
    del keep
    return ConfiguredCM(
        name=cm.name, M=M, W=int(s.W), flags=int(s.flags), clen=cm.clen,
        sttype=np.ascontiguousarray(cm.st.sttype, np.int8),
        stid=np.ascontiguousarray(cm.st.stid, np.int8),
        cfirst=np.ascontiguousarray(cm.st.cfirst, np.int32),
        cnum=np.ascontiguousarray(cm.st.cnum, np.int32),
        el_selfsc=float(s.el_selfsc), iel_selfsc=int(s.iel_selfsc),
        null=np.asarray(cm.null, np.float32), n3_omega=float(np.float32(cm.n3_omega)),
        **out,
    )


def cp9(cm: SynthCM) -> dict:
    """The CP9 HMM of a CM (cmgpu_prep_cp9; cp9_build_and_configure,
    src/cp9.rs:2212-2232): probabilities, integer scores and the HMM -> CM
    state map, as numpy arrays keyed by field name."""
    H = cm.clen
    p, keep = params_struct(cm)
    out = dict(mat=np.zeros((H + 1, 4), np.float32), ins=np.zeros((H + 1, 4), np.float32),
               t=np.zeros((H + 1, 10), np.float32), begin=np.zeros(H + 1, np.float32),
               end=np.zeros(H + 1, np.float32), msc=np.zeros((H + 1, 18), np.int32),
               isc=np.zeros((H + 1, 18), np.int32), otsc=np.zeros((H + 1, 12), np.int32),
               has_el=np.zeros(H + 1, np.uint8), hns2cs=np.zeros((H + 1, 3, 2), np.int32),
               el_pairs=np.zeros((cm.st.nodes, 2), np.int32))
    s = N.Cp9()
    s.M = H
    for k, ct in (("mat", C.c_float), ("ins", C.c_float), ("t", C.c_float), ("begin", C.c_float),
                  ("end", C.c_float), ("msc", C.c_int32), ("isc", C.c_int32), ("otsc", C.c_int32),
                  ("has_el", C.c_uint8), ("hns2cs", C.c_int32), ("el_pairs", C.c_int32)):
        setattr(s, k, N.ptr(out[k], ct))
    N.check(N.lib().cmgpu_prep_cp9(C.byref(p), C.byref(s)))
    del keep
    out["el_pairs"] = out["el_pairs"][: s.n_el]
    out["el_self"] = float(s.el_self)
    out["el_selfsc"] = int(s.el_selfsc)
    return out
