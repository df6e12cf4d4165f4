"""Seeded synthetic covariance models and sequences.

No CM file or `infernox-cmbuild` binary is available, so models are built
directly from a consensus secondary structure:

* ``structure(...)`` draws a consensus structure with a given number of
  consensus columns, base-paired fraction and bifurcation count.
* ``guide_tree(ct)`` builds the guide tree with the node rules of the
  reference's `hand_modelmaker` (src/cm_modelmaker.rs:729-975): END when the
  segment is empty, MATL when the left column is unpaired, MATR when the right
  one is, MATP when they pair with each other, otherwise BIF split at the
  helix boundary that best balances the two halves.
* ``cm_from_guide`` lays out states and child/parent links exactly as
  `cm_from_guide` (src/cm_modelmaker.rs:979-1110) does, so the scanner sees
  the same state graph a real CM of that structure has.
* Probabilities are seeded draws shaped like a built model: pair emissions
  concentrated on Watson-Crick/GU pairs (covariation), match emissions on a
  consensus residue, flat insert emissions (`flatten_insert_emissions`,
  src/cm_modelmaker.rs:2119), the END-adjacent dual insert detached
  (`cm_find_and_detach_dual_inserts`, src/cm_modelmaker.rs:1986-2070),
  EL self probability 0.94, PBEGIN/PEND 0.05, null3 omega 2^-16.

``emit(...)`` samples a homolog by walking the model from ROOT_S
(after src/cm_emit.rs:191-326), used for planting.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

# state / node codes (src/constants.rs:9-31)
D_ST, MP_ST, ML_ST, MR_ST, IL_ST, IR_ST, S_ST, E_ST, B_ST, EL_ST = range(10)
BIF_ND, MATP_ND, MATL_ND, MATR_ND, BEGL_ND, BEGR_ND, ROOT_ND, END_ND = range(8)
# unique state ids (src/constants.rs:46-81)
ROOT_S, ROOT_IL, ROOT_IR, BEGL_S, BEGR_S, BEGR_IL = 0, 1, 2, 3, 4, 5
MATP_MP, MATP_ML, MATP_MR, MATP_D, MATP_IL, MATP_IR = 6, 7, 8, 9, 10, 11
MATL_ML, MATL_D, MATL_IL, MATR_MR, MATR_D, MATR_IR = 12, 13, 14, 15, 16, 17
BIF_B, END_E = 18, 19

DEFAULT_EL_SELFPROB = 0.94
DEFAULT_PBEGIN = 0.05
DEFAULT_PEND = 0.05
DEFAULT_NULL3_OMEGA = 0.000015258791


def sre_log2(x: float) -> float:
    return math.log(x) * 1.44269504 if x > 0 else -1.0e36


# --------------------------------------------------------------------------
# consensus structures
# --------------------------------------------------------------------------

def _stem_cols(bp: int, inner: list, rng, bulge_rate: float) -> list:
    """A helix of `bp` pairs around `inner`, with occasional one-sided bulges."""
    left, right = [], []
    for k in range(bp):
        left.append("(")
        right.append(")")
        if k < bp - 1 and rng.random() < bulge_rate:
            if rng.random() < 0.5:
                left.append(".")
            else:
                right.append(".")
    return left + inner + right[::-1]


def structure(clen: int, paired_frac: float, nbif: int, seed: int,
              layout: str = "sidebyside") -> str:
    """Dot-bracket consensus structure with exactly `nbif` bifurcations.

    layout "sidebyside": nbif+1 hairpin stems in a row.
    layout "multibranch": one closing stem around a nbif+1-way multiloop.
    """
    rng = np.random.default_rng(seed)
    nstem = nbif + 1
    npair = max(nstem * 2, int(round(paired_frac * clen / 2)))
    if layout == "multibranch" and nbif > 0:
        nstem_inner = nbif + 1
        closing = max(2, npair // (nstem_inner + 1))
        rest = npair - closing
        inner_bp = [rest // nstem_inner + (1 if i < rest % nstem_inner else 0) for i in range(nstem_inner)]
    else:
        closing = 0
        inner_bp = [npair // nstem + (1 if i < npair % nstem else 0) for i in range(nstem)]
    unpaired = clen - 2 * npair
    loops = [max(3, 3 + int(rng.integers(0, 5))) for _ in inner_bp]
    free = unpaired - sum(loops)
    if free < 0:
        raise ValueError("clen too small for the requested pairs")
    # distribute the rest between linkers (nstem+1 slots) and bulges
    nlink = len(inner_bp) + 1
    link = [0] * nlink
    bulge_budget = int(free * 0.25)
    for _ in range(free - bulge_budget):
        link[int(rng.integers(0, nlink))] += 1
    bulge_rate = min(0.3, bulge_budget / max(1, npair))
    cols: list = ["."] * link[0]
    for s, bp in enumerate(inner_bp):
        cols += _stem_cols(bp, ["."] * loops[s], rng, bulge_rate)
        cols += ["."] * link[s + 1]
    if closing:
        body = cols
        cols = _stem_cols(closing, ["."] * 2 + body + ["."] * 2, rng, 0.0)
    ss = "".join(cols)
    # trim / pad unpaired columns to exactly clen
    while len(ss) > clen:
        k = ss.rfind(".")
        ss = ss[:k] + ss[k + 1:]
    while len(ss) < clen:
        ss = ss + "."
    return ss


def trna_like() -> str:
    """72 columns: a 7 bp closing stem around a four-way junction with three
    5 bp hairpins (two bifurcations)."""
    s = ("(((((((" + "." + "(((((" + "......" + ")))))" + "." +
         "(((((" + "......" + ")))))" + "...." + "(((((" + "......" + ")))))" +
         ")))))))" + "....")
    assert len(s) == 72
    return s


def ss_to_ct(ss: str) -> np.ndarray:
    """1-based partner array (0 = unpaired), like wuss2ct."""
    n = len(ss)
    ct = np.zeros(n + 1, dtype=np.int64)
    stack = []
    for i, c in enumerate(ss, start=1):
        if c in "(<[{":
            stack.append(i)
        elif c in ")>]}":
            j = stack.pop()
            ct[i], ct[j] = j, i
    if stack:
        raise ValueError("unbalanced structure")
    return ct


# --------------------------------------------------------------------------
# guide tree and state layout
# --------------------------------------------------------------------------

@dataclass
class GuideNode:
    type: int
    i: int
    j: int
    left: int = -1    # nxtl
    right: int = -1   # nxtr
    prv: int = -1


def guide_tree(ct: np.ndarray) -> list:
    """Preorder guide tree of hand_modelmaker for an all-consensus alignment."""
    n = len(ct) - 1
    nodes: list = []

    def add(parent: int, which: str, typ: int, i: int, j: int) -> int:
        k = len(nodes)
        nodes.append(GuideNode(typ, i, j, prv=parent))
        if parent >= 0:
            if which == "L":
                nodes[parent].left = k
            else:
                nodes[parent].right = k
        return k

    DUMMY = -1
    pda = [(-1, "L", 1, n, ROOT_ND)]
    while pda:
        parent, which, i, j, typ = pda.pop()
        if i > j:
            add(parent, which, END_ND, i, j)
        elif typ == ROOT_ND:
            v = add(parent, which, ROOT_ND, i, j)
            pda.append((v, "L", i, j, DUMMY))
        elif typ == BEGL_ND:
            v = add(parent, which, BEGL_ND, i, j)
            pda.append((v, "L", i, j, DUMMY))
        elif typ == BEGR_ND:
            v = add(parent, which, BEGR_ND, i, j)
            pda.append((v, "L", i, j, DUMMY))
        elif ct[i] == 0:
            v = add(parent, which, MATL_ND, i, j)
            pda.append((v, "L", i + 1, j, DUMMY))
        elif ct[j] == 0:
            v = add(parent, which, MATR_ND, i, j)
            pda.append((v, "L", i, j - 1, DUMMY))
        elif ct[i] == j:
            v = add(parent, which, MATP_ND, i, j)
            pda.append((v, "L", i + 1, j - 1, DUMMY))
        else:
            v = add(parent, which, BIF_ND, i, j)
            bestk, bestdiff = ct[i] + 1, n + 1
            k = ct[i] + 1
            while k <= ct[j]:
                diff = abs((k - i) - (j - k + 1))
                if diff < bestdiff:
                    bestdiff, bestk = diff, k
                while ct[k] == 0:
                    k += 1
                k = ct[k] + 1
            pda.append((v, "R", bestk, j, BEGR_ND))
            pda.append((v, "L", i, bestk - 1, BEGL_ND))
    return nodes


CHILD_COUNT = [1, 4, 2, 2, 1, 1, 0, 1]    # split-set size by next node type
PARENT_COUNT = [1, 6, 3, 3, 1, 2, 3, 0]   # states per node


@dataclass
class CMStructure:
    M: int
    nodes: int
    clen: int
    sttype: np.ndarray
    stid: np.ndarray
    ndidx: np.ndarray
    cfirst: np.ndarray
    cnum: np.ndarray
    plast: np.ndarray
    pnum: np.ndarray
    ndtype: np.ndarray
    nodemap: np.ndarray
    lpos: np.ndarray = field(default=None)  # consensus column of left emission per node


def cm_from_guide(g: list) -> CMStructure:
    nst = sum({BIF_ND: 1, MATP_ND: 6, MATL_ND: 3, MATR_ND: 3, BEGL_ND: 1, BEGR_ND: 2,
               ROOT_ND: 3, END_ND: 1}[x.type] for x in g)
    nnd = len(g)
    sttype = np.zeros(nst, np.int8)
    stid = np.zeros(nst, np.int8)
    ndidx = np.zeros(nst, np.int32)
    cfirst = np.zeros(nst, np.int32)
    cnum = np.zeros(nst, np.int32)
    plast = np.zeros(nst, np.int32)
    pnum = np.zeros(nst, np.int32)
    ndtype = np.zeros(nnd, np.int8)
    nodemap = np.zeros(nnd, np.int32)

    def ss(s, t, nd, sid, cf, cn, pl, pn):
        sttype[s], ndidx[s], stid[s], cfirst[s], cnum[s], plast[s], pnum[s] = t, nd, sid, cf, cn, pl, pn

    node = state = clen = 0
    pda = [0]
    while pda:
        v = pda.pop()
        x = g[v]
        nxt = g[x.left].type if x.left >= 0 else None
        prvt = g[x.prv].type if x.prv >= 0 else None
        nodemap[node] = state
        ndtype[node] = x.type
        if x.type == BIF_ND:
            ss(state, B_ST, node, BIF_B, state + 1, -1, state - 1, PARENT_COUNT[prvt])
            pda.append(state)
            state += 1
            node += 1
            pda.append(x.right)
            pda.append(x.left)
        elif x.type == MATP_ND:
            clen += 2
            cc = CHILD_COUNT[nxt]
            pc = PARENT_COUNT[prvt]
            ss(state, MP_ST, node, MATP_MP, state + 4, 2 + cc, state - 1, pc); state += 1
            ss(state, ML_ST, node, MATP_ML, state + 3, 2 + cc, state - 2, pc); state += 1
            ss(state, MR_ST, node, MATP_MR, state + 2, 2 + cc, state - 3, pc); state += 1
            ss(state, D_ST, node, MATP_D, state + 1, 2 + cc, state - 4, pc); state += 1
            ss(state, IL_ST, node, MATP_IL, state, 2 + cc, state, 5); state += 1
            ss(state, IR_ST, node, MATP_IR, state, 1 + cc, state, 6); state += 1
            node += 1
            pda.append(x.left)
        elif x.type in (MATL_ND, MATR_ND):
            clen += 1
            cc = CHILD_COUNT[nxt]
            pc = PARENT_COUNT[prvt]
            if x.type == MATL_ND:
                ss(state, ML_ST, node, MATL_ML, state + 2, 1 + cc, state - 1, pc); state += 1
                ss(state, D_ST, node, MATL_D, state + 1, 1 + cc, state - 2, pc); state += 1
                ss(state, IL_ST, node, MATL_IL, state, 1 + cc, state, 3); state += 1
            else:
                ss(state, MR_ST, node, MATR_MR, state + 2, 1 + cc, state - 1, pc); state += 1
                ss(state, D_ST, node, MATR_D, state + 1, 1 + cc, state - 2, pc); state += 1
                ss(state, IR_ST, node, MATR_IR, state, 1 + cc, state, 3); state += 1
            node += 1
            pda.append(x.left)
        elif x.type == BEGL_ND:
            ss(state, S_ST, node, BEGL_S, state + 1, CHILD_COUNT[nxt], state - 1, 1); state += 1
            node += 1
            pda.append(x.left)
        elif x.type == BEGR_ND:
            bifparent = pda.pop()
            cnum[bifparent] = state
            cc = CHILD_COUNT[nxt]
            ss(state, S_ST, node, BEGR_S, state + 1, 1 + cc, bifparent, 1); state += 1
            ss(state, IL_ST, node, BEGR_IL, state, 1 + cc, state, 2); state += 1
            node += 1
            pda.append(x.left)
        elif x.type == ROOT_ND:
            cc = CHILD_COUNT[nxt]
            ss(state, S_ST, node, ROOT_S, state + 1, 2 + cc, -1, 0); state += 1
            ss(state, IL_ST, node, ROOT_IL, state, 2 + cc, state, 2); state += 1
            ss(state, IR_ST, node, ROOT_IR, state, 1 + cc, state, 3); state += 1
            node += 1
            pda.append(x.left)
        elif x.type == END_ND:
            ss(state, E_ST, node, END_E, -1, 0, state - 1, PARENT_COUNT[prvt]); state += 1
            node += 1
    assert state == nst and node == nnd
    return CMStructure(nst, nnd, clen, sttype, stid, ndidx, cfirst, cnum, plast, pnum, ndtype, nodemap)


# --------------------------------------------------------------------------
# parameters
# --------------------------------------------------------------------------

PAIR_CONS = [(2, 1), (1, 2), (0, 3), (3, 0), (2, 3), (3, 2)]   # GC CG AU UA GU UG
PAIR_CONS_P = [0.3, 0.3, 0.15, 0.15, 0.05, 0.05]
WC_SET = {(2, 1), (1, 2), (0, 3), (3, 0), (2, 3), (3, 2)}


@dataclass
class SynthCM:
    """Probability-level CM plus the structure it was built from."""
    name: str
    ss: str
    st: CMStructure
    t: np.ndarray          # [M][6] float32
    e: np.ndarray          # [M][16] float32
    null: np.ndarray       # [4] float32
    el_selfsc: float
    pbegin: float = DEFAULT_PBEGIN
    pend: float = DEFAULT_PEND
    n3_omega: float = DEFAULT_NULL3_OMEGA

    @property
    def M(self) -> int:
        return self.st.M

    @property
    def clen(self) -> int:
        return self.st.clen


def _dirichlet_like(weights, rng, conc: float = 25.0) -> np.ndarray:
    w = np.asarray(weights, dtype=np.float64)
    g = rng.gamma(np.maximum(w * conc, 1e-3))
    g = g / g.sum()
    return g


def synth_cm(ss: str, seed: int, name: str = "synth", null=(0.25, 0.25, 0.25, 0.25),
             ins_open: float = 0.02, del_open: float = 0.03, ins_self: float = 0.35) -> SynthCM:
    rng = np.random.default_rng(seed)
    ct = ss_to_ct(ss)
    st = cm_from_guide(guide_tree(ct))
    M = st.M
    t = np.zeros((M, 6), np.float64)
    e = np.zeros((M, 16), np.float64)
    nullv = np.asarray(null, np.float64)
    for v in range(M):
        typ = st.sttype[v]
        # emissions
        if typ == MP_ST:
            cons = PAIR_CONS[rng.choice(len(PAIR_CONS), p=PAIR_CONS_P)]
            w = np.full(16, 0.15)
            for (a, b) in WC_SET:
                w[a * 4 + b] = 1.2
            w[cons[0] * 4 + cons[1]] = 14.0
            e[v] = _dirichlet_like(w / w.sum(), rng, 60.0)
        elif typ in (ML_ST, MR_ST):
            c = int(rng.integers(0, 4))
            w = np.full(4, 0.6)
            w[c] = 6.0
            e[v, :4] = _dirichlet_like(w / w.sum(), rng, 40.0)
        elif typ in (IL_ST, IR_ST):
            e[v, :4] = nullv
        # transitions
        if typ in (B_ST, E_ST):
            continue
        cf, cn = st.cfirst[v], st.cnum[v]
        kids = [cf + k for k in range(cn)]
        w = []
        for y in kids:
            ty = st.sttype[y]
            if ty in (IL_ST, IR_ST):
                w.append(ins_self if y == v else ins_open)
            elif ty == D_ST:
                w.append(0.25 if typ == D_ST else del_open)
            elif ty in (MP_ST, B_ST, E_ST):
                w.append(1.0)
            elif ty in (ML_ST, MR_ST):
                # ML/MR of a MATP node are half-deletions of the pair
                w.append(0.02 if st.stid[y] in (MATP_ML, MATP_MR) else 1.0)
            elif ty == S_ST:
                w.append(1.0)
            else:
                w.append(0.05)
        w = np.asarray(w)
        if typ in (IL_ST, IR_ST):
            w = w * np.where(np.asarray(kids) == v, 1.0, (1.0 - ins_self))
        t[v, :cn] = _dirichlet_like(w / w.sum(), rng, 30.0)
    # ROOT_S rarely enters the flanking inserts
    t[0, 0] *= 0.2
    t[0, 1] *= 0.2
    t[0, :st.cnum[0]] /= t[0, :st.cnum[0]].sum()
    t = t.astype(np.float32)
    e = e.astype(np.float32)
    _detach_dual_inserts(st, t)
    el = np.float32(sre_log2(DEFAULT_EL_SELFPROB))
    return SynthCM(name, ss, st, t, e, np.asarray(null, np.float32), float(el))


def _fnorm(row: np.ndarray, n: int) -> None:
    s = np.float32(0.0)
    for x in range(n):
        s = np.float32(s + row[x])
    if s != 0:
        for x in range(n):
            row[x] = np.float32(row[x] / s)
    else:
        row[:n] = np.float32(1.0 / n)


def emit_map(st: CMStructure):
    """Consensus bounds lpos/rpos per node (CreateEmitMap,
    src/cm_emitmap.rs:102-165)."""
    lpos = np.full(st.nodes, -1, np.int64)
    rpos = np.full(st.nodes, -1, np.int64)
    cpos = 0
    stack = [(False, 0)]
    while stack:
        on_right, nd = stack.pop()
        typ = st.ndtype[nd]
        if on_right:
            rpos[nd] = cpos + 1
            if typ in (MATP_ND, MATR_ND):
                cpos += 1
        else:
            if typ in (MATP_ND, MATL_ND):
                cpos += 1
            lpos[nd] = cpos
            stack.append((True, nd))
            if typ == BIF_ND:
                b = st.nodemap[nd]
                stack.append((False, int(st.ndidx[st.cnum[b]])))
                stack.append((False, int(st.ndidx[st.cfirst[b]])))
            elif typ != END_ND:
                stack.append((False, nd + 1))
    return lpos, rpos


def _detach_dual_inserts(st: CMStructure, t: np.ndarray) -> None:
    """Where a left and a right insert state map to the same consensus gap,
    the one followed by an END state loses every transition into it
    (cm_find_and_detach_dual_inserts / cm_detach_state,
    src/cm_modelmaker.rs:1986-2071)."""
    lpos, rpos = emit_map(st)
    clen = int(rpos[0] - 1)
    lins = [-1] * (clen + 1)
    rins = [-1] * (clen + 1)
    lins[0] = 1
    rins[clen] = 2
    for nd in range(st.nodes):
        v = int(st.nodemap[nd])
        typ = st.ndtype[nd]
        if typ == MATP_ND:
            lins[lpos[nd]] = v + 4
            rins[rpos[nd] - 1] = v + 5
        elif typ == MATL_ND:
            lins[lpos[nd]] = v + 2
        elif typ == MATR_ND:
            rins[rpos[nd] - 1] = v + 2
        elif typ == BEGR_ND:
            lins[lpos[nd]] = v + 1
    for cc in range(clen + 1):
        a, b = lins[cc], rins[cc]
        if a == -1 or b == -1:
            continue
        if st.sttype[a + 1] == E_ST:
            d = a
        elif st.sttype[b + 1] == E_ST:
            d = b
        else:
            continue
        x_offset = 0 if st.sttype[d] == IL_ST else 1
        y = st.pnum[d] - 1
        while y >= 1:
            xp = st.plast[d] - y
            t[xp, x_offset] = 0.0
            _fnorm(t[xp], st.cnum[xp])
            y -= 1


# --------------------------------------------------------------------------
# sequences
# --------------------------------------------------------------------------

def random_dsq(n: int, gc: float, rng) -> np.ndarray:
    """i.i.d. residues 0..3 with the given GC fraction."""
    p = np.array([(1 - gc) / 2, gc / 2, gc / 2, (1 - gc) / 2])
    return rng.choice(4, size=n, p=p).astype(np.uint8)


def emit(cm: SynthCM, rng, max_len: int = 100000) -> np.ndarray:
    """Sample a homolog from the global model (ROOT_S downwards)."""
    st = cm.st

    def expand(v0: int) -> list:
        res: list = []
        v = v0
        right: list = []
        while True:
            typ = st.sttype[v]
            if typ == E_ST:
                break
            if typ == B_ST:
                res += expand(st.cfirst[v])
                res += expand(st.cnum[v])
                break
            if typ == MP_ST:
                k = rng.choice(16, p=cm.e[v] / cm.e[v].sum())
                res.append(k // 4)
                right.append(k % 4)
            elif typ in (ML_ST, IL_ST):
                res.append(int(rng.choice(4, p=cm.e[v, :4] / cm.e[v, :4].sum())))
            elif typ in (MR_ST, IR_ST):
                right.append(int(rng.choice(4, p=cm.e[v, :4] / cm.e[v, :4].sum())))
            cn = st.cnum[v]
            p = cm.t[v, :cn].astype(np.float64)
            v = st.cfirst[v] + int(rng.choice(cn, p=p / p.sum()))
            if len(res) + len(right) > max_len:
                break
        return res + right[::-1]
    return np.asarray(expand(0), np.uint8)


def revcomp(dsq: np.ndarray) -> np.ndarray:
    """Bottom strand: reverse order, canonical codes complemented as 3-x
    (src/cm_search.rs:1823-1827)."""
    r = dsq[::-1].copy()
    m = r < 4
    r[m] = 3 - r[m]
    return r


def hb_band_rects(st: CMStructure, p: int, i0: int, j0: int, slack: int, rng):
    """Per-state (i, j) rectangles of HMM-band shape for a homolog whose
    consensus column 1 sits at sequence position p: state v of node n spans
    i near p + lpos(n) - 1 and j near p + rpos(n) - 1, widened by a seeded
    0..slack on each side and clipped to the envelope [i0, j0]; END states
    sit one residue left of their i (empty subsequences).  Returns imin,
    imax, jmin, jmax, ready for hb.ij2d_bands."""
    lpos, rpos = emit_map(st)
    M = st.M
    node = np.asarray(st.ndidx, np.int64)
    ic = p + lpos[node] - 1
    jc = p + rpos[node] - 1
    emits_left = np.isin(np.asarray(st.sttype), (1, 2, 4))  # MP, ML, IL: i is their own column
    ic = np.where(emits_left, ic, ic + 1)
    jc = np.maximum(jc, ic - 1)
    s = lambda: rng.integers(0, slack + 1, M)
    imin = np.clip(ic - s(), i0, j0)
    imax = np.clip(ic + s(), i0, j0)
    jmin = np.clip(jc - s(), i0, j0)
    jmax = np.clip(jc + s(), i0, j0)
    is_end = np.asarray(st.sttype) == 7
    jmin = np.where(is_end, np.clip(ic - 1 - slack, i0 - 1, j0), jmin)
    jmax = np.where(is_end, np.clip(ic - 1 + slack, i0 - 1, j0), jmax)
    imin = np.minimum(imin, imax)
    jmax = np.maximum(jmax, jmin)
    return imin.astype(np.int32), imax.astype(np.int32), jmin.astype(np.int32), jmax.astype(np.int32)
