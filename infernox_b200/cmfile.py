"""CM files: the reader of the reference's ASCII save format and a writer of
the same format for this package's models.

``read_cm(text_or_path)`` restates `cm_file_read_from_reader_opt`
(src/cm_file.rs:51-914): the INFERNAL1/a (v1.1) and INFERNAL-1 (v1.0)
headers, node and state lines (plast / pnum / cfirst / cnum verbatim, the
v1.1 QDB band columns), log-odds scores turned back into probabilities with
`ascii2prob` (:943-952, exp(x / 1.44269504) * null in double, rounded to
float), the renormalisation of every distribution (`cm_renormalize`,
:1029-1045, esl_vec_FNorm with Kahan sums in float), the v1.0 detachment of
END-adjacent dual inserts, W from the file or the model, and the unique
state ids.  The HMMER3/f filter block after the CM (`P7Profile::parse_hmmer3`,
src/p7_hmm.rs:172-560) becomes a `p7.P7Profile` with its composition and
local E-value parameters.  Configuration (local begins and ends) is the
scanner's own step (`model.configure`), as `cm_file_read_global` leaves it.

``write_cm(cm, ...)`` writes a model in the INFERNAL1/a layout of
`cm_file_write_ascii` (src/cm_file.rs:1297-1518): scores as `prob2ascii`
(`%.3f` of log2(p / null)), six transition columns, the NULL line against
the uniform background; with a p7 profile it appends a HMMER3/f block.
"""
from __future__ import annotations

import ctypes
import ctypes.util
import math
import os
from dataclasses import dataclass, field

import numpy as np

from . import p7 as P7
from .synth import (B_ST, BEGL_ND, BEGR_ND, BIF_ND, CMStructure, D_ST, E_ST, EL_ST, END_ND, IL_ST, IR_ST,
                    MATL_ND, MATP_ND, MATR_ND, ML_ST, MP_ST, MR_ST, ROOT_ND, S_ST, SynthCM, _detach_dual_inserts)

STATE_TYPES = {"D": D_ST, "MP": MP_ST, "ML": ML_ST, "MR": MR_ST, "IL": IL_ST, "IR": IR_ST, "S": S_ST, "E": E_ST,
               "B": B_ST, "EL": EL_ST}
NODE_TYPES = {"BIF": BIF_ND, "MATP": MATP_ND, "MATL": MATL_ND, "MATR": MATR_ND, "BEGL": BEGL_ND, "BEGR": BEGR_ND,
              "ROOT": ROOT_ND, "END": END_ND}
STATE_NAMES = {v: k for k, v in STATE_TYPES.items()}
NODE_NAMES = {v: k for k, v in NODE_TYPES.items()}

# unique state id of (node type, state type), Infernal's DeriveUniqueStateCode
# (src/cm_file.rs:1124-1175)
_STID = {
    (ROOT_ND, S_ST): 0, (ROOT_ND, IL_ST): 1, (ROOT_ND, IR_ST): 2, (BEGL_ND, S_ST): 3, (BEGR_ND, S_ST): 4,
    (BEGR_ND, IL_ST): 5, (MATP_ND, MP_ST): 6, (MATP_ND, ML_ST): 7, (MATP_ND, MR_ST): 8, (MATP_ND, D_ST): 9,
    (MATP_ND, IL_ST): 10, (MATP_ND, IR_ST): 11, (MATL_ND, ML_ST): 12, (MATL_ND, D_ST): 13, (MATL_ND, IL_ST): 14,
    (MATR_ND, MR_ST): 15, (MATR_ND, D_ST): 16, (MATR_ND, IR_ST): 17, (BIF_ND, B_ST): 18, (END_ND, E_ST): 19,
}

_libm = ctypes.CDLL(ctypes.util.find_library("m") or "libm.so.6")
_libm.expf.restype = ctypes.c_float
_libm.expf.argtypes = [ctypes.c_float]
_libm.powf.restype = ctypes.c_float
_libm.powf.argtypes = [ctypes.c_float, ctypes.c_float]
_libm.logf.restype = ctypes.c_float
_libm.logf.argtypes = [ctypes.c_float]

F32 = np.float32


def ascii2prob(s: str, null: float) -> np.float32:
    """src/cm_file.rs:943-952."""
    if s == "*":
        return F32(0.0)
    return F32(math.exp(float(s) / 1.44269504) * float(F32(null)))


def prob2ascii(p: float, null: float) -> str:
    """src/cm_file.rs:1213-1219: '*' for 0, else %.3f of log2(p / null)
    (the division in float, the logarithm in double)."""
    if F32(p) == 0:
        return "*"
    return "%.3f" % (math.log(float(F32(F32(p) / F32(null)))) * 1.44269504)


def _fnorm(v: np.ndarray) -> None:
    """esl_vec_FNorm in float with a Kahan sum (src/cm_file.rs:954-989)."""
    s = F32(0.0)
    c = F32(0.0)
    for x in v:
        y = F32(x - c)
        t = F32(s + y)
        c = F32(F32(t - s) - y)
        s = t
    if s != 0:
        for q in range(len(v)):
            v[q] = F32(v[q] / s)
    else:
        v[:] = F32(1.0) / F32(len(v))


@dataclass
class CMFile:
    """One model of a CM file: the probability-level CM, the file's header
    values, the band columns of a v1.1 file and the p7 filter (if any)."""
    cm: SynthCM
    version: str
    W: int
    acc: str = None
    desc: str = None
    w_beta: float = 1e-7
    qdb_beta1: float = 1e-7
    qdb_beta2: float = 1e-15
    n2_omega: float = 0.03125
    cutoffs: dict = field(default_factory=dict)      # GA / TC / NC
    exp: dict = field(default_factory=dict)          # ECMGC / ECMGI / ECMLC / ECMLI -> 6 values
    efp7gf: tuple = None
    bands: dict = field(default_factory=dict)        # dmin1 / dmax1 / dmin2 / dmax2 (v1.1)
    p7: P7.P7Profile = None
    p7_compo: np.ndarray = None
    p7_evparam: dict = field(default_factory=dict)   # lmmu, lmlambda, lvmu, lvlambda, lftau, lflambda
    p7_max_length: int = 0


def _text(src) -> str:
    if isinstance(src, bytes):
        return src.decode()
    if "\n" not in src and os.path.exists(src):
        with open(src) as fh:
            return fh.read()
    return src


def read_cm(src) -> CMFile:
    """The first model of a CM file (a path or the file's text)."""
    models = read_cms(src, limit=1)
    if not models:
        raise ValueError("no CM in the input")
    return models[0]


def _format(line: str) -> str:
    """parse_format_line (src/cm_file.rs:916-941): '1.1' or '1.0'."""
    s = line.strip()
    if s.startswith("INFERNAL1/a"):
        return "1.1"
    if s.startswith("INFERNAL-1") or s.startswith("INFERNAL1"):
        if "1.0" in s:
            return "1.0"
        if "1.1" in s:
            return "1.1"
        return "1.0"
    raise ValueError(f"not a CM file format line: {line!r}")


def read_cms(src, limit: int = 0) -> list:
    """Every model of a CM file (at most `limit` when > 0)."""
    lines = _text(src).splitlines()
    out, at = [], 0
    while at < len(lines) and (limit <= 0 or len(out) < limit):
        if not lines[at].strip():
            at += 1
            continue
        m, at = _read_one(lines, at)
        out.append(m)
    return out


def _read_one(lines, at):
    fmt = _format(lines[at])
    at += 1
    h = dict(name="", acc=None, desc=None, M=0, nodes=0, clen=0, W=0, el_selfsc=0.0, pbegin=0.05, pend=0.05,
             w_beta=1e-7, qdb_beta1=1e-7, qdb_beta2=1e-15, n2_omega=0.03125, n3_omega=0.03125, efp7gf=None)
    null = [F32(0.0)] * 4
    cut, exp = {}, {}
    while at < len(lines):
        raw = lines[at]
        line = raw.strip()
        at += 1
        if line.startswith("MODEL:") or line.startswith("CM"):
            break
        parts = line.split()
        if not parts:
            continue
        tag, rest = parts[0], line[len(parts[0]):].strip()
        if tag == "NAME" and len(parts) >= 2:
            h["name"] = parts[1]
        elif tag in ("STATES", "NODES", "CLEN") and len(parts) >= 2:
            h[{"STATES": "M", "NODES": "nodes", "CLEN": "clen"}[tag]] = int(parts[1])
        elif tag == "ELSELF" and len(parts) >= 2:
            h["el_selfsc"] = float(F32(float(parts[1])))
        elif tag in ("GA", "TC", "NC") and len(parts) >= 2:
            cut[tag] = float(F32(float(parts[1])))
        elif tag == "NULL":
            for i in range(min(4, len(parts) - 1)):
                null[i] = F32(F32(0.25) * _libm.powf(2.0, float(F32(float(parts[i + 1])))))
        elif tag == "W" and len(parts) >= 2:
            h["W"] = int(parts[1])
        elif tag in ("PBEGIN", "PEND") and len(parts) >= 2:
            h[tag.lower()] = float(F32(float(parts[1])))
        elif tag in ("WBETA", "QDBBETA1", "QDBBETA2", "N2OMEGA", "N3OMEGA") and len(parts) >= 2:
            h[{"WBETA": "w_beta", "QDBBETA1": "qdb_beta1", "QDBBETA2": "qdb_beta2", "N2OMEGA": "n2_omega",
               "N3OMEGA": "n3_omega"}[tag]] = float(parts[1])
        elif tag == "EFP7GF" and len(parts) >= 3:
            h["efp7gf"] = (float(parts[1]), float(parts[2]))
        elif tag in ("ECMLC", "ECMGC", "ECMLI", "ECMGI") and len(parts) >= 7:
            exp[tag] = tuple(float(x) for x in parts[1:7])
        elif tag in ("E-LC", "E-GC", "E-LI", "E-GI") and len(parts) >= 8:
            exp["ECM" + tag[2:]] = tuple(float(x) for x in (parts[2], parts[3], parts[4], parts[5], parts[6],
                                                            parts[7]))
        elif tag == "ACC" and len(parts) >= 2:
            h["acc"] = parts[1]
        elif tag == "DESC":
            h["desc"] = rest
    M, nodes = h["M"], h["nodes"]
    if M <= 0 or nodes <= 0:
        raise ValueError("CM file: STATES and NODES must be positive")
    if all(x == 0 for x in null):
        null = [F32(0.25)] * 4
    sttype = np.zeros(M, np.int8)
    stid = np.zeros(M, np.int8)
    ndidx = np.zeros(M, np.int32)
    cfirst = np.zeros(M, np.int32)
    cnum = np.zeros(M, np.int32)
    plast = np.zeros(M, np.int32)
    pnum = np.zeros(M, np.int32)
    ndtype = np.zeros(nodes, np.int8)
    nodemap = np.zeros(nodes, np.int32)
    seen = np.zeros(nodes, bool)
    t = np.zeros((M, 6), np.float32)
    e = np.zeros((M, 16), np.float32)
    bands = {k: np.zeros(M, np.int32) for k in ("dmin1", "dmax1", "dmin2", "dmax2")}
    node = -1
    mincols = 10 if fmt == "1.1" else 6
    while at < len(lines):
        line = lines[at].strip()
        at += 1
        if line == "//":
            break
        if not line:
            continue
        b0, b1 = line.find("["), line.find("]")
        if b0 >= 0 and b1 > b0:
            inner = line[b0 + 1:b1].split()
            if len(inner) >= 2 and inner[0] in NODE_TYPES:
                node = int(inner[1])
                if 0 <= node < nodes:
                    ndtype[node] = NODE_TYPES[inner[0]]
            continue
        parts = line.split()
        if len(parts) < mincols or parts[0] not in STATE_TYPES:
            continue
        st = STATE_TYPES[parts[0]]
        v = int(parts[1])
        if not 0 <= v < M:
            continue
        plast[v], pnum[v], cfirst[v], cnum[v] = int(parts[2]), int(parts[3]), int(parts[4]), int(parts[5])
        col = 6
        if fmt == "1.1":
            bands["dmin2"][v], bands["dmin1"][v], bands["dmax1"][v], bands["dmax2"][v] = (int(x) for x in parts[6:10])
            col = 10
        sttype[v], ndidx[v] = st, node
        if 0 <= node < nodes and not seen[node]:
            nodemap[node] = v
            seen[node] = True
        for k in range(min(max(int(cnum[v]), 0), 6)):
            if col < len(parts):
                t[v, k] = ascii2prob(parts[col], 1.0)
                col += 1
        ne = 16 if st == MP_ST else (4 if st in (ML_ST, MR_ST, IL_ST, IR_ST) else 0)
        for idx in range(ne):
            if col < len(parts):
                nl = F32(null[idx // 4] * null[idx % 4]) if st == MP_ST else null[idx]
                e[v, idx] = ascii2prob(parts[col], nl)
                col += 1
    for v in range(M):
        stid[v] = _STID.get((int(ndtype[ndidx[v]]), int(sttype[v])), 0)
    clen = h["clen"]
    struct = CMStructure(M, nodes, clen, sttype, stid, ndidx, cfirst, cnum, plast, pnum, ndtype, nodemap)
    if fmt == "1.0":
        _detach_dual_inserts(struct, t)
    # cm_renormalize (src/cm_file.rs:1029-1045)
    nullv = np.array(null, np.float32)
    _fnorm(nullv)
    for v in range(M):
        if cnum[v] > 0 and sttype[v] != B_ST:
            row = t[v, :cnum[v]].copy()
            _fnorm(row)
            t[v, :cnum[v]] = row
        if sttype[v] in (ML_ST, MR_ST, IL_ST, IR_ST):
            row = e[v, :4].copy()
            _fnorm(row)
            e[v, :4] = row
        elif sttype[v] == MP_ST:
            row = e[v].copy()
            _fnorm(row)
            e[v] = row
    cm = SynthCM(h["name"], "", struct, t, e, nullv, h["el_selfsc"], pbegin=h["pbegin"], pend=h["pend"],
                 n3_omega=float(F32(h["n3_omega"])))
    W = h["W"] if h["W"] > 0 else 0
    res = CMFile(cm, fmt, W, acc=h["acc"], desc=h["desc"], w_beta=h["w_beta"], qdb_beta1=h["qdb_beta1"],
                 qdb_beta2=h["qdb_beta2"], n2_omega=h["n2_omega"], cutoffs=cut, exp=exp, efp7gf=h["efp7gf"],
                 bands=bands if fmt == "1.1" else {})
    # the p7 filter block (HMMER3/f), when the model carries one
    while at < len(lines):
        s = lines[at].strip()
        if s.startswith("HMMER3"):
            at = _read_hmmer3(lines, at + 1, res)
            break
        if s.startswith("INFERNAL") or s == "//":
            break
        at += 1
    return res, at


def _nexp(s: str) -> np.float32:
    """-score -> probability in float (expf(-x), '*' = 0)."""
    if s == "*":
        return F32(0.0)
    return F32(_libm.expf(float(-F32(float(s)))))


def _read_hmmer3(lines, at, res: CMFile) -> int:
    """P7Profile::parse_hmmer3 (src/p7_hmm.rs:172-560): header, COMPO, node 0
    and the M nodes (match emissions, insert emissions, transitions)."""
    m, maxl, ev = 0, 0, {}
    while at < len(lines):
        line = lines[at].strip()
        at += 1
        if line.startswith("HMM "):
            break
        if line.startswith("//"):
            return at
        parts = line.split()
        if not parts:
            continue
        if parts[0] == "LENG":
            m = int(parts[1])
        elif parts[0] == "MAXL":
            maxl = int(parts[1])
        elif parts[0] == "STATS" and len(parts) >= 5 and parts[1] == "LOCAL":
            key = {"MSV": ("lmmu", "lmlambda"), "VITERBI": ("lvmu", "lvlambda"),
                   "FORWARD": ("lftau", "lflambda")}.get(parts[2])
            if key:
                ev[key[0]], ev[key[1]] = float(parts[3]), float(parts[4])
    if m <= 0:
        return at
    mat = np.zeros((m + 1, 4), np.float32)
    trans = np.zeros((m + 1, 7), np.float32)
    compo = np.full(4, 0.25, np.float32)
    at += 1  # the transition header line
    parts = lines[at].split() if at < len(lines) else []
    if len(parts) >= 5 and parts[0] == "COMPO":
        compo = np.array([_nexp(x) for x in parts[1:5]], np.float32)
        at += 1
    at += 1  # node-0 insert emissions
    parts = lines[at].split() if at < len(lines) else []
    if len(parts) >= 7:
        trans[0] = [_nexp(x) for x in parts[:7]]
    at += 1
    for k in range(1, m + 1):
        if at >= len(lines):
            break
        mline = lines[at].split()
        if mline and mline[0].startswith("//"):
            break
        if len(mline) >= 5:
            mat[k] = [_nexp(x) for x in mline[1:5]]
        tl = lines[at + 2].split() if at + 2 < len(lines) else []
        if len(tl) >= 7:
            trans[k] = [_nexp(x) for x in tl[:7]]
        at += 3
    while at < len(lines) and lines[at].strip() != "//":
        at += 1
    res.p7 = P7.P7Profile(m, mat, trans)
    res.p7_compo = compo
    res.p7_evparam = ev
    res.p7_max_length = maxl
    return at + 1


def _g(x: float) -> str:
    return "%g" % x


def _printprob(p: float) -> str:
    """printprob (src/p7_hmm.rs:560-575): -ln(p) to 5 decimals, '*' for 0."""
    p = F32(p)
    if p == 0:
        return "*"
    if p == 1:
        return "0.00000"
    return "%.5f" % float(-F32(_libm.logf(float(p))))


def write_cm(cm: SynthCM, p7: P7.P7Profile = None, compo=None, evparam: dict = None, max_length: int = 0) -> str:
    """The model in the INFERNAL1/a layout (src/cm_file.rs:1297-1518), with
    W and the QDB band columns from the library's own band engine, and the
    p7 filter as a HMMER3/f block when given."""
    from . import model as MD
    g = MD.configure(cm, local=False)
    st = cm.st
    M, K = st.M, 4
    null = np.asarray(cm.null, np.float32)
    o = ["INFERNAL1/a [1.1.5 | Sep 2023]", f"NAME     {cm.name or 'cm'}", f"STATES   {M}", f"NODES    {st.nodes}",
         f"CLEN     {st.clen}", f"W        {g.W}", "ALPH     RNA", "RF       no", "CONS     no", "MAP      no",
         f"PBEGIN   {_g(float(F32(cm.pbegin)))}", f"PEND     {_g(float(F32(cm.pend)))}", "WBETA    1e-07",
         "QDBBETA1 1e-07", "QDBBETA2 1e-15", f"N2OMEGA  {_g(0.000015258791):>6}",
         f"N3OMEGA  {_g(float(F32(cm.n3_omega))):>6}", f"ELSELF   {float(F32(cm.el_selfsc)):.8f}", "NSEQ     0",
         "EFFN     0.000000",
         "NULL    " + "".join(f"{prob2ascii(null[x], 0.25):>6} " for x in range(K)), "CM"]
    for v in range(M):
        nd = int(st.ndidx[v])
        if int(st.nodemap[nd]) == v:
            o.append(f"{'':>45}[ {NODE_NAMES[int(st.ndtype[nd])]:<4} {nd:>4} ] {'-':>6} {'-':>6} - - - -")
        row = (f"    {STATE_NAMES[int(st.sttype[v])]:>2} {v:>5} {int(st.plast[v]):>5} {int(st.pnum[v]):>1} "
               f"{int(st.cfirst[v]):>5} {int(st.cnum[v]):>5} {int(g.dmin2[v]):>5} {int(g.dmin1[v]):>5} "
               f"{int(g.dmax1[v]):>5} {int(g.dmax2[v]):>5} ")
        x = 0
        if st.sttype[v] != B_ST:
            for x in range(int(st.cnum[v])):
                row += f"{prob2ascii(cm.t[v][x], 1.0):>7} "
            x = int(st.cnum[v])
        row += f"{'':>7} " * (6 - x)
        if st.sttype[v] == MP_ST:
            row += "".join(f"{prob2ascii(cm.e[v][a * K + b], F32(null[a] * null[b])):>6} "
                           for a in range(K) for b in range(K))
        elif st.sttype[v] in (ML_ST, MR_ST, IL_ST, IR_ST):
            row += "".join(f"{prob2ascii(cm.e[v][a], null[a]):>6} " for a in range(K))
        o.append(row)
    o.append("//")
    if p7 is not None:
        ev = evparam or {}
        m = p7.M
        mat = np.asarray(p7.mat, np.float32).reshape(m + 1, 4)
        tr = np.asarray(p7.trans, np.float32).reshape(m + 1, 7)
        comp = np.full(4, 0.25, np.float32) if compo is None else np.asarray(compo, np.float32)
        o += ["HMMER3/f [3.1b2 | February 2015]", f"NAME  {cm.name or 'cm'}", f"LENG  {m}",
              f"MAXL  {max_length or 2 * m}", "ALPH  rna", "RF    no", "MM    no", "CONS  no", "CS    no",
              "MAP   no",
              f"STATS LOCAL MSV      {ev.get('lmmu', 0.0):8.4f} {ev.get('lmlambda', 0.0):8.5f}",
              f"STATS LOCAL VITERBI  {ev.get('lvmu', 0.0):8.4f} {ev.get('lvlambda', 0.0):8.5f}",
              f"STATS LOCAL FORWARD  {ev.get('lftau', 0.0):8.4f} {ev.get('lflambda', 0.0):8.5f}",
              "HMM          A        C        G        U",
              "            m->m     m->i     m->d     i->m     i->i     d->m     d->d",
              "  COMPO   " + "  ".join(f"{_printprob(x):>7}" for x in comp),
              "          " + "  ".join(f"{_printprob(0.25):>7}" for _ in range(4)),
              "          " + "  ".join(f"{_printprob(x):>7}" for x in tr[0])]
        for k in range(1, m + 1):
            o.append(f"{k:>7}   " + "  ".join(f"{_printprob(x):>7}" for x in mat[k]) + f" {k:>6} - - - -")
            o.append("          " + "  ".join(f"{_printprob(0.25):>7}" for _ in range(4)))
            o.append("          " + "  ".join(f"{_printprob(x):>7}" for x in tr[k]))
        o.append("//")
    return "\n".join(o) + "\n"
