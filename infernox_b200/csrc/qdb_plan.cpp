// Builds the device plan (qdb_plan.h) of a configured CM for one semiring
// and band set, and counts the exact DP work of a scan.
//
// Band selection and per-state dn/dxcap follow generic_scan
// (src/cm_nohmm.rs:431-456); the d = 0 base values follow the reference's
// scan-matrix initialisation (src/cm_nohmm.rs:489-537); el_sca is built by
// repeated addition (src/cm_nohmm.rs:471-474).
#include <algorithm>
#include <cstring>
#include <string>

#include "../../include/cmscan_gpu.h"
#include "cm_internal.h"
#include "qdb_plan.h"
#include "sweep_plan.h"

namespace cmx {

void set_error(const std::string &msg);

namespace {

inline uint32_t fbits(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    return u;
}
inline float bitsf(uint32_t u) {
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}
inline int32_t wadd(int32_t a, int32_t b) { return (int32_t)((uint32_t)a + (uint32_t)b); }

struct Bands {
    std::vector<int32_t> dmin, dmax, dn, dxcap;
};

Bands select_bands(const cmgpu_cm *cm, int qdbidx) {
    Bands b;
    const int M = cm->M, W = cm->W;
    b.dmin.resize(M);
    b.dmax.resize(M);
    b.dn.resize(M);
    b.dxcap.resize(M);
    for (int v = 0; v < M; v++) {
        if (qdbidx == CMGPU_NOQDB) {
            b.dmin[v] = 0;
            b.dmax[v] = W;
        } else if (qdbidx == CMGPU_QDB1) {
            b.dmin[v] = cm->dmin1[v];
            b.dmax[v] = cm->dmax1[v];
        } else {
            b.dmin[v] = cm->dmin2[v];
            b.dmax[v] = cm->dmax2[v];
        }
        int base = cm->sttype[v] == MP_ST ? 2 : 1;
        int dn = std::max(b.dmin[v], base);
        if (dn > W) dn = W;
        b.dn[v] = dn;
        b.dxcap[v] = std::min(b.dmax[v], W);
    }
    return b;
}

}  // namespace

bool build_plan(const cmgpu_cm *cm, int semiring, int qdbidx, Plan &p) {
    const int M = cm->M, W = cm->W;
    if (M < 2 || W < 1 || M > 32767 || W > 32000) {
        set_error("model too large for the scan plan (M <= 32767, W <= 32000)");
        return false;
    }
    const bool inside = semiring == CMGPU_INSIDE_I32;
    p = Plan();
    p.M = M;
    p.W = W;
    p.semiring = semiring;
    p.qdbidx = qdbidx;
    p.local = (cm->flags & (1u << 10)) != 0;
    Bands b = select_bands(cm, qdbidx);

    const uint32_t ZERO = inside ? (uint32_t)(-INFTY) : fbits(IMPOSSIBLE);
    auto add = [&](uint32_t a, uint32_t c) -> uint32_t {
        if (inside) return (uint32_t)wadd((int32_t)a, (int32_t)c);
        return fbits(bitsf(a) + bitsf(c));
    };
    auto vmax = [&](uint32_t a, uint32_t c) -> uint32_t {
        if (inside) return (int32_t)a >= (int32_t)c ? a : c;
        return bitsf(a) >= bitsf(c) ? a : c;
    };
    auto possible_bits = [&](uint32_t x) -> bool {
        // not_impossible(scbits(x)) (src/cm_nohmm.rs:20-22, :148-150)
        if (inside) {
            int32_t s = (int32_t)x;
            if (s == -INFTY) return false;
            float f = (float)((double)s / INTSCALE);
            return f > IMPOSSIBLE + 1.0f;
        }
        return bitsf(x) > IMPOSSIBLE + 1.0f;
    };
    auto begin_possible = [&](uint32_t x) -> bool {
        // Sr::is_possible: NOT_IMPOSSIBLE for f32, != -INFTY for i32
        if (inside) return (int32_t)x != -INFTY;
        return bitsf(x) > IMPOSSIBLE + 1.0f;
    };

    // score tables
    p.tsc.assign((size_t)M * MAXC, ZERO);
    p.endsc.assign(M, ZERO);
    p.beginsc_all.assign(M, ZERO);
    p.esc.assign((size_t)M * ESC, ZERO);
    for (int v = 0; v < M; v++) {
        for (int x = 0; x < MAXC; x++)
            p.tsc[(size_t)v * MAXC + x] = inside ? (uint32_t)cm->itsc[(size_t)v * MAXC + x]
                                                 : fbits(cm->tsc[(size_t)v * MAXC + x]);
        p.endsc[v] = inside ? (uint32_t)cm->iendsc[v] : fbits(cm->endsc[v]);
        p.beginsc_all[v] = inside ? (uint32_t)cm->ibeginsc[v] : fbits(cm->beginsc[v]);
        for (int x = 0; x < ESC; x++)
            p.esc[(size_t)v * ESC + x] =
                inside ? (uint32_t)cm->ioesc[(size_t)v * ESC + x] : fbits(cm->oesc[(size_t)v * ESC + x]);
    }
    // compact canonical emission table (codes 0..3) for shared memory
    p.escoff.assign(M, -1);
    p.esc_c.clear();
    for (int v = 0; v < M; v++) {
        int st = cm->sttype[v];
        if (st == MP_ST) {
            p.escoff[v] = (int32_t)p.esc_c.size();
            for (int a = 0; a < 4; a++)
                for (int c2 = 0; c2 < 4; c2++) p.esc_c.push_back(p.esc[(size_t)v * ESC + a * KP + c2]);
        } else if (st == ML_ST || st == MR_ST || st == IL_ST || st == IR_ST) {
            p.escoff[v] = (int32_t)p.esc_c.size();
            for (int a = 0; a < 4; a++) p.esc_c.push_back(p.esc[(size_t)v * ESC + a]);
        }
    }
    const uint32_t el_self = inside ? (uint32_t)cm->iel_selfsc : fbits(cm->el_selfsc);
    p.el_sca.assign((size_t)W + 1, 0u);
    p.el_sca[0] = inside ? 0u : fbits(0.0f);
    for (int d = 1; d <= W; d++) p.el_sca[d] = add(p.el_sca[d - 1], el_self);

    // d = 0 base values (src/cm_nohmm.rs:489-537)
    p.init0.assign(M, ZERO);
    for (int v = M - 1; v >= 0; v--) {
        int st = cm->sttype[v];
        if (st == E_ST) {
            p.init0[v] = inside ? 0u : fbits(0.0f);
        } else if (st == S_ST || st == D_ST) {  // includes BEGL_S
            uint32_t a0 = p.endsc[v];
            for (int yo = 0; yo < cm->cnum[v]; yo++)
                a0 = vmax(a0, add(p.init0[cm->cfirst[v] + yo], p.tsc[(size_t)v * MAXC + yo]));
            a0 = vmax(a0, ZERO);
            p.init0[v] = a0;
        } else if (st == B_ST) {
            p.init0[v] = add(p.init0[cm->cfirst[v]], p.init0[cm->cnum[v]]);
        } else {
            p.init0[v] = ZERO;
        }
    }

    // per-state metadata
    p.states.assign(M, StateDev());
    std::vector<int> width(M, 0);
    for (int v = 0; v < M; v++) {
        StateDev &s = p.states[v];
        int st = cm->sttype[v];
        s.type = (uint8_t)st;
        s.flags = 0;
        s.cnum = (uint8_t)(st == B_ST ? 2 : cm->cnum[v]);
        s.sd = (uint8_t)state_delta(st);
        s.dn = (int16_t)b.dn[v];
        s.dxcap = (int16_t)b.dxcap[v];
        s.escoff = p.escoff[v];
        width[v] = std::max(0, b.dxcap[v] - b.dn[v] + 1);
        if (st == E_ST || v == 0) width[v] = 0;  // E cells are constants; ROOT_S is never read
        if (cm->stid[v] == BEGL_S) s.flags |= SF_BEGL;
        if (right_emitter(st)) s.flags |= SF_TWO_SLOT;
        if (possible_bits(p.endsc[v])) s.flags |= SF_ENDSC;
        if (p.local && v >= 1 && begin_possible(p.beginsc_all[v])) s.flags |= SF_BEGIN;
    }
    // index range every state's deck must cover: own band + all reads
    std::vector<int> lo(M, 1 << 30), hi(M, -1);
    auto cover = [&](int y, int a, int c) {
        if (c < a) return;
        lo[y] = std::min(lo[y], a);
        hi[y] = std::max(hi[y], c);
    };
    for (int v = 0; v < M; v++) {
        if (width[v] > 0) cover(v, b.dn[v], b.dxcap[v]);
        int st = cm->sttype[v];
        if (st == E_ST) continue;
        if (v == 0) {
            for (int yo = 0; yo < cm->cnum[0]; yo++) cover(cm->cfirst[0] + yo, b.dn[0], b.dxcap[0]);
            continue;
        }
        if (width[v] <= 0) continue;
        if (st == B_ST) {
            int wl = cm->cfirst[v], y = cm->cnum[v];
            cover(y, std::max(0, std::min(b.dmin[y], W)), std::min(b.dmax[y], W));
            cover(wl, std::max(0, std::min(b.dmin[wl], W)), std::min(b.dmax[wl], W));
        } else {
            int sd = state_delta(st);
            for (int yo = 0; yo < cm->cnum[v]; yo++) cover(cm->cfirst[v] + yo, b.dn[v] - sd, b.dxcap[v] - sd);
        }
    }
    // deck layout
    std::vector<int32_t> base(M, 0);
    int64_t off = 0;
    for (int v = 0; v < M; v++) {
        StateDev &s = p.states[v];
        if (hi[v] < lo[v]) {
            s.span = 0;
            continue;
        }
        int span = hi[v] - lo[v] + 1;
        s.span = span;
        int64_t slots = (s.flags & SF_BEGL) ? (int64_t)W + 1 : (s.flags & SF_TWO_SLOT) ? 2 : 1;
        base[v] = (int32_t)(off - lo[v]);
        if (lo[v] <= 0 && 0 <= hi[v] && p.init0[v] != ZERO)
            for (int64_t q = 0; q < slots; q++) {
                p.init_off.push_back((int32_t)(base[v] + q * span));
                p.init_val.push_back(p.init0[v]);
            }
        off += slots * span;
        if (off > ((int64_t)1 << 30)) {
            set_error("deck exceeds 2^30 cells");
            return false;
        }
    }
    p.deck_elems = off;
    // own write bases and child read bases by column parity
    p.wb.assign((size_t)M * 2, 0);
    p.cb.assign((size_t)M * 12, 0);
    auto slot_base = [&](int y, int slot) -> int32_t {
        const StateDev &s = p.states[y];
        return base[y] + ((s.flags & SF_TWO_SLOT) ? slot * s.span : 0);
    };
    for (int v = 0; v < M; v++) {
        int st = cm->sttype[v];
        for (int par = 0; par < 2; par++) p.wb[(size_t)v * 2 + par] = slot_base(v, par);
        if (st == E_ST) continue;
        if (st == B_ST) {
            int wl = cm->cfirst[v], y = cm->cnum[v];
            int32_t *c = &p.cb[(size_t)v * 12];
            c[0] = c[1] = base[wl];
            c[2] = c[3] = base[y];
            c[4] = std::min(b.dmin[y], W);
            c[5] = std::min(b.dmax[y], W);
            c[6] = std::min(b.dmin[wl], W);
            c[7] = std::min(b.dmax[wl], W);
            c[8] = p.states[wl].span;
            continue;
        }
        bool rem = right_emitter(st);
        int sd = v == 0 ? 0 : state_delta(st);
        for (int yo = 0; yo < cm->cnum[v]; yo++) {
            int y = cm->cfirst[v] + yo;
            for (int par = 0; par < 2; par++) {
                int slot = rem ? (par ^ 1) : par;  // prv for right emitters, cur otherwise
                p.cb[(size_t)v * 12 + yo * 2 + par] = slot_base(y, slot) - sd;
            }
        }
    }
    p.root_dn = b.dn[0];
    p.root_dxcap = b.dxcap[0];
    p.root_cnum = cm->cnum[0];
    for (int v = 1; v < M; v++) {
        if (!(p.states[v].flags & SF_BEGIN)) continue;
        BeginDev bd;
        bd.v = v;
        if (p.states[v].flags & SF_BEGL) {
            bd.base0 = bd.base1 = base[v];
        } else {
            bd.base0 = slot_base(v, 0);
            bd.base1 = slot_base(v, 1);
        }
        bd.dn = (int16_t)b.dn[v];
        bd.dxcap = (int16_t)b.dxcap[v];
        if (width[v] <= 0) continue;
        p.begins.push_back(bd);
        p.beginsc.push_back(p.beginsc_all[v]);
    }

    // levels: right emitters read only the previous column -> level 0; every
    // other state sits one level above its deepest same-column child.
    std::vector<int> level(M, -1);
    int nlev = 1;
    for (int v = M - 1; v >= 1; v--) {
        int st = cm->sttype[v];
        if (st == E_ST) continue;
        if (right_emitter(st)) {
            level[v] = 0;
            continue;
        }
        int lv = 1;
        if (st == B_ST) {
            lv = std::max(lv, level[cm->cfirst[v]] + 1);
            lv = std::max(lv, level[cm->cnum[v]] + 1);
        } else {
            for (int yo = 0; yo < cm->cnum[v]; yo++) {
                int y = cm->cfirst[v] + yo;
                if (y == v || cm->sttype[y] == E_ST) continue;
                lv = std::max(lv, level[y] + 1);
            }
        }
        level[v] = lv;
        nlev = std::max(nlev, lv + 1);
    }
    p.level_start.assign(1, 0);
    p.chunks.clear();
    for (int l = 0; l < nlev; l++) {
        std::vector<std::pair<double, ChunkDev>> lc;
        for (int v = 1; v < M; v++) {
            if (level[v] != l) continue;
            const StateDev &s = p.states[v];
            if (width[v] <= 0) continue;
            int st = s.type;
            if (st == IL_ST) {
                lc.push_back({1e9 + width[v], ChunkDev{v, -1}});
            } else {
                for (int d0 = s.dn; d0 <= s.dxcap; d0 += 64) {
                    double cost = st == B_ST ? 1e6 + d0 : (double)s.cnum;
                    lc.push_back({cost, ChunkDev{v, d0}});
                }
            }
        }
        std::stable_sort(lc.begin(), lc.end(),
                         [](const std::pair<double, ChunkDev> &a, const std::pair<double, ChunkDev> &c) {
                             return a.first > c.first;
                         });
        for (auto &x : lc) p.chunks.push_back(x.second);
        p.max_level_chunks = std::max(p.max_level_chunks, (int)lc.size());
        p.level_start.push_back((int32_t)p.chunks.size());
    }
    return true;
}

// Exact cells / terms of one column at row limit jrow, counted the way the
// oracle's counters count them.
void count_column(const cmgpu_cm *cm, const Plan &p, const Bands &b, int jrow, double &cells, double &terms) {
    const int M = cm->M, W = cm->W;
    for (int v = 1; v < M; v++) {
        int st = cm->sttype[v];
        if (st == E_ST) continue;
        int dn = b.dn[v], dx = std::min(jrow, b.dxcap[v]);
        if (dx < dn) continue;
        int n = dx - dn + 1;
        cells += n;
        if (st == B_ST) {
            int wl = cm->cfirst[v], y = cm->cnum[v];
            int dn_y = std::min(b.dmin[y], W), dx_y = std::min(b.dmax[y], W);
            int dn_w = std::min(b.dmin[wl], W), dx_w = std::min(b.dmax[wl], W);
            for (int d = dn; d <= dx; d++) {
                int kmin = std::max(0, std::max(dn_y, d - dx_w));
                int kmax = std::min(dx_y, d - dn_w);
                if (kmax >= kmin) terms += kmax - kmin + 1;
            }
        } else {
            terms += (double)n * cm->cnum[v];
        }
    }
    int dn0 = b.dn[0], dx0 = std::min(jrow, b.dxcap[0]);
    if (dx0 >= dn0) {
        cells += dx0 - dn0 + 1;
        terms += (double)(dx0 - dn0 + 1) * cm->cnum[0];
        for (const BeginDev &bd : p.begins) {
            int y = bd.v;
            int dn = std::max(dn0, b.dn[y]);
            int dx = std::min(dx0, std::min(jrow, b.dxcap[y]));
            if (dx >= dn) terms += dx - dn + 1;
        }
    }
}

void count_column_public(const cmgpu_cm *cm, const Plan &p, int qdbidx, int jrow, double &cells, double &terms) {
    Bands b = select_bands(cm, qdbidx);
    count_column(cm, p, b, jrow, cells, terms);
}

bool count_work(const cmgpu_cm *cm, int semiring, int qdbidx, int64_t L, double &cells, double &terms) {
    Plan p;
    if (!build_plan(cm, semiring, qdbidx, p)) return false;
    Bands b = select_bands(cm, qdbidx);
    cells = terms = 0;
    const int W = cm->W;
    int64_t warm = std::min<int64_t>(L, W - 1);
    for (int64_t j = 1; j <= warm; j++) count_column(cm, p, b, (int)j, cells, terms);
    if (L > warm) {
        double c = 0, t = 0;
        count_column(cm, p, b, W, c, t);
        cells += c * (double)(L - warm);
        terms += t * (double)(L - warm);
    }
    return true;
}

// ---------------------------------------------------------------------------
// sweep plan
// ---------------------------------------------------------------------------
namespace {

// unique state ids (src/constants.rs:46-81)
enum {
    UID_ROOT_S = 0, UID_ROOT_IL, UID_ROOT_IR, UID_BEGL_S, UID_BEGR_S, UID_BEGR_IL, UID_MATP_MP, UID_MATP_ML,
    UID_MATP_MR, UID_MATP_D, UID_MATP_IL, UID_MATP_IR, UID_MATL_ML, UID_MATL_D, UID_MATL_IL, UID_MATR_MR,
    UID_MATR_D, UID_MATR_IR, UID_BIF_B, UID_END_E
};

struct NodeShape {
    int type, nst, nsplit;  // node type, states, split (non-insert) states
    int ids[6];             // unique state ids in state order
};

// The node a state id starts, with its state list (src/cm_modelmaker.rs:979-1110).
bool node_shape(int first_id, NodeShape &ns) {
    switch (first_id) {
    case UID_ROOT_S: ns = {ROOT_ND, 3, 1, {UID_ROOT_S, UID_ROOT_IL, UID_ROOT_IR}}; return true;
    case UID_BEGL_S: ns = {BEGL_ND, 1, 1, {UID_BEGL_S}}; return true;
    case UID_BEGR_S: ns = {BEGR_ND, 2, 1, {UID_BEGR_S, UID_BEGR_IL}}; return true;
    case UID_MATP_MP:
        ns = {MATP_ND, 6, 4, {UID_MATP_MP, UID_MATP_ML, UID_MATP_MR, UID_MATP_D, UID_MATP_IL, UID_MATP_IR}};
        return true;
    case UID_MATL_ML: ns = {MATL_ND, 3, 2, {UID_MATL_ML, UID_MATL_D, UID_MATL_IL}}; return true;
    case UID_MATR_MR: ns = {MATR_ND, 3, 2, {UID_MATR_MR, UID_MATR_D, UID_MATR_IR}}; return true;
    case UID_BIF_B: ns = {BIF_ND, 1, 1, {UID_BIF_B}}; return true;
    case UID_END_E: ns = {END_ND, 1, 1, {UID_END_E}}; return true;
    default: return false;
    }
}

}  // namespace

bool build_sweep_plan(const cmgpu_cm *cm, const Plan &p, int qdbidx, SweepPlan &sp, std::string *why) {
    auto fail = [&](const std::string &m) {
        if (why) *why = m;
        return false;
    };
    const int M = cm->M, W = cm->W;
    if (W + 1 > SW_MAX_S) return fail("W above the sweep kernel's limit");
    sp = SweepPlan();
    sp.M = M;
    sp.W = W;
    sp.S = ((W + 1 + 31) / 32) * 32;
    sp.RW = W + 1;
    Bands b = select_bands(cm, qdbidx);

    // nodes from the unique state ids
    std::vector<NodeShape> shape;
    std::vector<int> v0s, node_of(M, -1);
    for (int v = 0; v < M;) {
        NodeShape ns;
        if (!node_shape(cm->stid[v], ns)) return fail("state list does not start a node where expected");
        if (v + ns.nst > M) return fail("truncated node");
        for (int q = 0; q < ns.nst; q++) {
            if (cm->stid[v + q] != ns.ids[q]) return fail("unexpected state order inside a node");
            node_of[v + q] = (int)shape.size();
        }
        shape.push_back(ns);
        v0s.push_back(v);
        v += ns.nst;
    }
    const int nn = (int)shape.size();
    if (nn > 32767 || M > 32767) return fail("model too large");
    if (shape[0].type != ROOT_ND) return fail("first node is not ROOT");

    // children: own inserts, then the split states of node n+1
    auto is_insert = [&](int v) { return cm->sttype[v] == IL_ST || cm->sttype[v] == IR_ST; };
    std::vector<int> bif_of_begl(M, -1), bif_of_begr(M, -1);
    for (int v = 0; v < M; v++) {
        const int st = cm->sttype[v], n = node_of[v];
        if (st == E_ST) continue;
        if (st == B_ST) {
            int wl = cm->cfirst[v], y = cm->cnum[v];
            if (wl != v + 1 || cm->stid[wl] != UID_BEGL_S || y <= v || y >= M || cm->stid[y] != UID_BEGR_S)
                return fail("bifurcation children are not BEGL_S / BEGR_S");
            SwBif bf{};
            bf.kdn_y = (int16_t)std::min(b.dmin[y], W);
            bf.kdx_y = (int16_t)std::min(b.dmax[y], W);
            bf.kdn_w = (int16_t)std::min(b.dmin[wl], W);
            bf.kdx_w = (int16_t)std::min(b.dmax[wl], W);
            bf.begl = (int16_t)wl;
            bf.begr = (int16_t)y;
            bf.b = (int16_t)v;
            bif_of_begl[wl] = bif_of_begr[y] = (int)sp.bifs.size();
            sp.bifs.push_back(bf);
            continue;
        }
        if (n + 1 >= nn) return fail("a non-END last node");
        std::vector<int> kids;
        const int v0 = v0s[n];
        for (int q = 0; q < shape[n].nst; q++) {
            int u = v0 + q;
            if (!is_insert(u)) continue;
            if (is_insert(v) && u < v) continue;  // an insert's children start at itself
            kids.push_back(u);
        }
        for (int q = 0; q < shape[n + 1].nsplit; q++) kids.push_back(v0s[n + 1] + q);
        if ((int)kids.size() != cm->cnum[v] || kids[0] != cm->cfirst[v])
            return fail("children are not the node's inserts followed by the next node's split states");
    }
    if (sp.bifs.size() > 255) return fail("too many bifurcations");

    // cell ranges: own band plus every index a reader uses (as build_plan)
    std::vector<int> lo(M, 1 << 30), hi(M, -1);
    auto cover = [&](int y, int a, int c) {
        if (c < a) return;
        lo[y] = std::min(lo[y], a);
        hi[y] = std::max(hi[y], c);
    };
    for (int v = 0; v < M; v++) {
        const int st = cm->sttype[v];
        const int width = std::max(0, b.dxcap[v] - b.dn[v] + 1);
        if (st == E_ST) continue;
        if (v == 0) {
            for (int yo = 0; yo < cm->cnum[0]; yo++) cover(cm->cfirst[0] + yo, b.dn[0], b.dxcap[0]);
            continue;
        }
        if (width <= 0) continue;
        cover(v, b.dn[v], b.dxcap[v]);
        if (st == B_ST) {
            int wl = cm->cfirst[v], y = cm->cnum[v];
            cover(y, std::max(0, std::min(b.dmin[y], W)), std::min(b.dmax[y], W));
            cover(wl, std::max(0, std::min(b.dmin[wl], W)), std::min(b.dmax[wl], W));
        } else {
            const int sd = state_delta(st);
            for (int yo = 0; yo < cm->cnum[v]; yo++) cover(cm->cfirst[v] + yo, b.dn[v] - sd, b.dxcap[v] - sd);
        }
    }

    // per-state metadata
    sp.st.assign(M, SwState());
    for (int v = 0; v < M; v++) {
        const StateDev &sd = p.states[v];
        SwState &s = sp.st[v];
        s.lo = (int16_t)(hi[v] >= lo[v] ? lo[v] : 1);
        s.hi = (int16_t)(hi[v] >= lo[v] ? hi[v] : 0);
        s.dn = sd.dn;
        s.dxcap = sd.dxcap;
        s.type = sd.type;
        s.flags = sd.flags & (SF_ENDSC | SF_BEGIN);
        s.cnum = sd.cnum;
        s.sd = sd.sd;
        if (sd.escoff > 32767) return fail("emission table too large");
        s.escoff = (int16_t)sd.escoff;
        s.slot = (uint8_t)(v - v0s[node_of[v]]);
        if (v == 0) s.flags |= SWF_ROOT;
        if (cm->stid[v] == UID_BEGL_S) s.flags |= SWF_BEGL;
        if (cm->stid[v] == UID_BEGR_S) s.flags |= SWF_BEGR;
    }

    // previous-column reads, deck slots and child locations
    sp.kid.assign((size_t)M * MAXC, 0);
    sp.nodes.assign(nn, SwNode());
    int64_t deck = 0;
    for (int n = 0; n < nn; n++) {
        SwNode &nd = sp.nodes[n];
        const int v0 = v0s[n];
        nd.type = (uint8_t)shape[n].type;
        nd.nst = (uint8_t)shape[n].nst;
        nd.v0 = (int16_t)v0;
        nd.io0 = (int16_t)sp.io.size();
        nd.aux = 0;
        if (shape[n].type == BIF_ND) {
            for (size_t k = 0; k < sp.bifs.size(); k++)
                if (sp.bifs[k].b == v0) nd.aux = (uint8_t)k;
        } else if (shape[n].type == BEGL_ND) {
            nd.aux = (uint8_t)bif_of_begl[v0];
        } else if (shape[n].type == BEGR_ND) {
            nd.aux = (uint8_t)bif_of_begr[v0];
        }
        std::vector<int> prev;  // states read in the previous column, ascending
        for (int q = 0; q < shape[n].nst; q++) {
            const int v = v0 + q, st = cm->sttype[v];
            if (!right_emitter(st)) continue;
            for (int yo = 0; yo < cm->cnum[v]; yo++) prev.push_back(cm->cfirst[v] + yo);
        }
        std::sort(prev.begin(), prev.end());
        prev.erase(std::unique(prev.begin(), prev.end()), prev.end());
        if (prev.size() > (size_t)SW_SLOTS) return fail("too many previous-column reads in one node");
        for (size_t k = 0; k < prev.size(); k++) {
            const int y = prev[k];
            if (cm->stid[y] == UID_BEGL_S || cm->stid[y] == UID_BEGR_S)
                return fail("a right emitter reads a subtree start state");
            SwIO e{};
            e.y = (int16_t)y;
            e.pslot = (uint8_t)k;
            e.cur = node_of[y] == n ? (uint8_t)(y - v0) : (uint8_t)(8 + y - v0s[n + 1]);
            e.lo = sp.st[y].lo;
            e.hi = sp.st[y].hi;
            e.deck = (int32_t)deck;
            deck += sp.S;
            sp.io.push_back(e);
        }
        nd.nio = (uint8_t)prev.size();
        for (int q = 0; q < shape[n].nst; q++) {
            const int v = v0 + q, st = cm->sttype[v];
            if (st == E_ST || st == B_ST) continue;
            for (int yo = 0; yo < cm->cnum[v]; yo++) {
                const int y = cm->cfirst[v] + yo;
                uint8_t code;
                if (right_emitter(st)) {
                    size_t k = std::find(prev.begin(), prev.end(), y) - prev.begin();
                    code = (uint8_t)(KID_PREV * 8 + k);
                } else if (node_of[y] == n) {
                    code = (uint8_t)(KID_OWN * 8 + (y - v0));
                } else {
                    code = (uint8_t)(KID_NEXT * 8 + (y - v0s[n + 1]));
                }
                sp.kid[(size_t)v * MAXC + yo] = code;
            }
        }
    }
    if (deck > ((int64_t)1 << 30)) return fail("deck too large");
    sp.deck_words = deck;
    sp.ring_words = (int64_t)sp.bifs.size() * sp.RW * sp.S;
    return true;
}

}  // namespace cmx

extern "C" int cmgpu_count_work(const cmgpu_cm *cm, int semiring, int qdbidx, int32_t L, double *cells,
                                double *terms) {
    if (!cm || !cells || !terms || L < 0) return CMGPU_EINVAL;
    double c = 0, t = 0;
    if (L > 0 && !cmx::count_work(cm, semiring, qdbidx, L, c, t)) return CMGPU_EINVAL;
    *cells = c;
    *terms = t;
    return CMGPU_OK;
}
