// Node-sweep QDB-banded CYK / Inside window scanner for sm_100a.
//
// One warp owns one work item (a piece of a window plus W-1 warm-up columns,
// as in qdb_scan.cu) and computes every cell of a column itself, walking the
// CM's nodes from the last to the first; warps share nothing but the model
// tables, so a column needs no CTA barrier at all.
//
// Why a node at a time: the children of a state of node n are node n's own
// insert states and the split states of node n+1 (cm_from_guide,
// src/cm_modelmaker.rs:979-1110).  So while node n runs, the only current-
// column values it reads are its own and those of node n+1: two node buffers
// of six state slots in shared memory hold them, swapping roles every node.
// Right emitters (MP, MR, IR) read the previous column instead
// (jp_y = prv, src/cm_nohmm.rs:575): the states they read keep a slot in the
// warp's deck in global memory; while node n+1 runs, cp.async copies node
// n's slots into one of two previous-column buffers, and after node n ran
// its current values overwrite them.
// A bifurcation reads its BEGR_S from a per-warp row in shared memory and its
// BEGL_S from a ring of W+1 columns in global memory (alpha_begl,
// src/cm_nohmm.rs:578-600).  Local begins are a MAX (src/cm_nohmm.rs:
// 700-746): each begin state folds its cells into a per-warp ROOT row as it
// computes them.
//
// Cells are evaluated with the reference's operand order: reduce_c_order for
// emitters, S and D states, natural child order for BEGL_S, plain order for
// ROOT_S, ascending k for bifurcations, and the IL self-loop chain resolved
// exactly by the blocked fixed-point iteration of qdb_scan.cu.  Within a
// state, lanes take cells d, d+32, ... (IL: consecutive blocks), and a
// __syncwarp separates states.
#include <cuda_runtime.h>
#include <climits>
#include <cstdint>

#include "devbuf.h"
#include "semiring.cuh"
#include "sweep_kernel.h"

namespace cmx {
namespace swdev {

using dev::Sem;
using dev::IMPOSSIBLE_D;
using dev::reduce_c;
using dev::reduce_c_noself;

#ifndef SW_NC
#define SW_NC 2
#endif

constexpr unsigned FULL = 0xffffffffu;

// Integer Inside with ILogsum (src/cp9.rs:65-75) written without branches:
// the cases that add nothing (min at -INFTY, difference beyond the table)
// index the zero entry the kernel stores at tbl[nz].
struct SemInsBF : Sem<true> {
    __device__ static __forceinline__ int32_t comb(int32_t a, int32_t b, const uint16_t *tbl, int nz) {
        const int32_t mx0 = max(a, b), mn = min(a, b);
        const uint32_t diff = (uint32_t)mx0 - (uint32_t)mn;
        const int32_t mx = max(mx0, -dev::INFTY_D);
        const uint32_t idx = mn <= -dev::INFTY_D ? (uint32_t)nz : min(diff, (uint32_t)nz);
        return (int32_t)((uint32_t)mx + (uint32_t)tbl[idx]);
    }
};
#ifdef SW_COMB_BRANCHY
template <bool INS> struct SemSel { typedef Sem<INS> type; };
#else
template <bool INS> struct SemSel { typedef Sem<false> type; };
template <> struct SemSel<true> { typedef SemInsBF type; };
#endif
constexpr int B_ST_D = 8, E_ST_D = 7, IL_ST_D = 4;  // sttype codes (cm_internal.h)

struct St {  // unpacked SwState
    int lo, hi, dn, dxcap, type, flags, cnum, sd, escoff, slot;
};

__device__ __forceinline__ St unpack(int4 q) {
    St s;
    s.lo = (int16_t)(q.x & 0xffff);
    s.hi = (int16_t)((uint32_t)q.x >> 16);
    s.dn = (int16_t)(q.y & 0xffff);
    s.dxcap = (int16_t)((uint32_t)q.y >> 16);
    s.type = q.z & 0xff;
    s.flags = (q.z >> 8) & 0xff;
    s.cnum = (q.z >> 16) & 0xff;
    s.sd = ((uint32_t)q.z >> 24) & 0xff;
    s.escoff = (int16_t)(q.w & 0xffff);
    s.slot = (q.w >> 16) & 0xff;
    return s;
}

struct Ctx {
    const SweepParams *p;
    const int4 *st;
    const uint8_t *kid;
    const uint32_t *tsc, *endsc, *init0, *bsv, *escc, *el;
    const uint16_t *tbl;
    const int4 *nodes, *io, *bifs;
    int nz;
    uint32_t *buf;    // two node buffers (12 S), then two previous-column buffers (12 S)
    uint32_t *begr;   // nbif rows of S
    uint32_t *bmax;   // S: local-begin maxima of the current column
    uint8_t *ring;    // residues
    int rmask;
    uint32_t *deck;   // this warp's deck slots (global)
    uint32_t *rings;  // this warp's BEGL rings (global)
    int S, RW, lane;
    int rdn, rdx;     // ROOT_S band: the cells a local begin can reach
};

struct Col {
    int j, jrow, jm, resj, item, jreport;
    bool first;
};

template <class Sm>
__device__ __forceinline__ typename Sm::T esc1(const Ctx &c, int v, int escoff, int x) {
    if (x < 4) return Sm::ld(c.escc + escoff + x);
    return Sm::ldg(c.p->esc + v * 324 + x);
}
template <class Sm>
__device__ __forceinline__ typename Sm::T esc2(const Ctx &c, int v, int escoff, int a, int b) {
    if ((a | b) < 4) return Sm::ld(c.escc + escoff + a * 4 + b);
    return Sm::ldg(c.p->esc + v * 324 + a * 18 + b);
}

// Base of a child's current-column cells (code = kind * 8 + slot); pb is
// the previous-column buffer of the node being computed.
__device__ __forceinline__ const uint32_t *kid_base(const Ctx &c, int code, int par, int pb) {
    const int kind = code >> 3, slot = code & 7;
    const int buf = kind == KID_PREV ? 12 + pb * SW_SLOTS : ((kind == KID_OWN ? par : par ^ 1) * SW_SLOTS);
    return c.buf + (buf + slot) * c.S;
}

// Asynchronous 4-byte copy global -> shared (cp.async, sm_80+).
__device__ __forceinline__ void cp_async4(uint32_t *dst, const uint32_t *src) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// Local begin (MAX into the ROOT row) of a begin state's cell d.
template <class Sm>
__device__ __forceinline__ void begin_fold(const Ctx &c, int d, typename Sm::T x, typename Sm::T bsc) {
    typedef typename Sm::T T;
    if (d < c.rdn || d > c.rdx) return;
    const T cand = Sm::add(x, bsc);
    const T b = Sm::ld(c.bmax + d);
    if (b < cand) Sm::st(c.bmax + d, cand);
}

// reduce_c (reduce_c_order for Inside, any bracketing for CYK) of NC
// independent cells at once: one switch on cnum, the NC fold chains side by
// side inside each case so that their latencies overlap.
template <class Sm, int NC>
__device__ __forceinline__ void reduce_n(int cnum, const typename Sm::T (&t)[NC][6], const typename Sm::T (&init)[NC],
                                         typename Sm::T (&o)[NC], const uint16_t *tb, int nz) {
#define CB(a, b) Sm::comb(a, b, tb, nz)
    if (!Sm::ORDERED) {
#pragma unroll
        for (int q = 0; q < NC; q++) o[q] = reduce_c<Sm>(cnum, t[q], init[q], tb, nz);
        return;
    }
    switch (cnum) {
    case 1:
#pragma unroll
        for (int q = 0; q < NC; q++) o[q] = CB(init[q], t[q][0]);
        break;
    case 2:
#pragma unroll
        for (int q = 0; q < NC; q++) o[q] = CB(CB(t[q][1], init[q]), t[q][0]);
        break;
    case 3:
#pragma unroll
        for (int q = 0; q < NC; q++) o[q] = CB(CB(CB(t[q][2], t[q][1]), init[q]), t[q][0]);
        break;
    case 4:
#pragma unroll
        for (int q = 0; q < NC; q++) o[q] = CB(CB(CB(CB(t[q][3], t[q][2]), init[q]), t[q][1]), t[q][0]);
        break;
    case 5:
#pragma unroll
        for (int q = 0; q < NC; q++)
            o[q] = CB(CB(CB(CB(CB(t[q][4], t[q][3]), init[q]), t[q][1]), t[q][2]), t[q][0]);
        break;
    case 6:
#pragma unroll
        for (int q = 0; q < NC; q++)
            o[q] = CB(CB(CB(CB(CB(CB(t[q][5], init[q]), t[q][4]), t[q][3]), t[q][2]), t[q][1]), t[q][0]);
        break;
    default:  // cnum is 1..6 for every non-B, non-E state of a CM
#pragma unroll
        for (int q = 0; q < NC; q++) o[q] = init[q];
    }
#undef CB
}

// An ordinary state (not E, B, IL, ROOT_S): cells lo..hi, band cells
// computed, the rest the fill of the reference's decks.  Two cells per lane
// per step (d and d+32), evaluated side by side.
template <class Sm>
__device__ __forceinline__ void do_plain(const Ctx &c, const Col &C, int v, const St &s, int par, int pb,
                                         uint32_t *dst) {
    typedef typename Sm::T T;
    const T ZERO = Sm::zero();
    const uint32_t *kp[6];
    T ts[6];
#pragma unroll
    for (int yo = 0; yo < 6; yo++) {
        kp[yo] = c.buf;
        ts[yo] = ZERO;
        if (yo < s.cnum) {
            kp[yo] = kid_base(c, c.kid[v * 6 + yo], par, pb) - s.sd;
            ts[yo] = Sm::ld(c.tsc + v * 6 + yo);
        }
    }
    const bool endsc = s.flags & SF_ENDSC;
    const T es = endsc ? Sm::ld(c.endsc + v) : ZERO;
    const bool begin = s.flags & SF_BEGIN;
    const T bsc = begin ? Sm::ld(c.bsv + v) : ZERO;
    const T base0 = Sm::ld(c.init0 + v);
    const int dx = min(C.jrow, s.dxcap);
    const bool natural = s.flags & SWF_BEGL;  // BEGL_S folds its children in natural order
    const int t = s.type;
    const T ej = (t == 3 || t == 5) ? esc1<Sm>(c, v, s.escoff, C.resj) : ZERO;
    // computed cells: [clo, chi] = band within the written range
    const int clo = max(s.lo, s.dn), chi = min(s.hi, dx);
    constexpr int NC = SW_NC;
    for (int d0 = s.lo; d0 <= s.hi; d0 += 32 * NC) {
        int dd[NC];
        bool live[NC], inb[NC];
        T terms[NC][6], init[NC], sc[NC];
#pragma unroll
        for (int q = 0; q < NC; q++) {
            dd[q] = d0 + c.lane + 32 * q;
            live[q] = dd[q] <= s.hi;
            inb[q] = dd[q] >= clo && dd[q] <= chi;
            // cells outside the band are evaluated at a band cell (discarded)
            const int e = chi >= clo ? min(max(dd[q], clo), chi) : s.dn;
#pragma unroll
            for (int yo = 0; yo < 6; yo++) terms[q][yo] = ZERO;
            if (chi >= clo) {
#pragma unroll
                for (int yo = 0; yo < 6; yo++)
                    if (yo < s.cnum) terms[q][yo] = Sm::add(Sm::ld(kp[yo] + e), ts[yo]);
                init[q] = endsc ? Sm::add(Sm::ld(c.el + e - s.sd), es) : ZERO;
            } else {
                init[q] = ZERO;
            }
        }
        if (chi >= clo) {
            if (natural) {
#pragma unroll
                for (int q = 0; q < NC; q++) {
                    sc[q] = init[q];
#pragma unroll
                    for (int yo = 0; yo < 6; yo++)
                        if (yo < s.cnum) sc[q] = Sm::comb(sc[q], terms[q][yo], c.tbl, c.nz);
                }
            } else {
                reduce_n<Sm, NC>(s.cnum, terms, init, sc, c.tbl, c.nz);
            }
#pragma unroll
            for (int q = 0; q < NC; q++) {
                const int e = min(max(dd[q], clo), chi);
                if (t == 2 || t == 4) {  // ML, IL: residue i = j-d+1
                    sc[q] = Sm::add(sc[q], esc1<Sm>(c, v, s.escoff, c.ring[(C.j - e + 1) & c.rmask]));
                } else if (t == 3 || t == 5) {  // MR, IR: residue j
                    sc[q] = Sm::add(sc[q], ej);
                } else if (t == 1) {  // MP
                    sc[q] = Sm::add(sc[q], esc2<Sm>(c, v, s.escoff, c.ring[(C.j - e + 1) & c.rmask], C.resj));
                }
            }
        }
#pragma unroll
        for (int q = 0; q < NC; q++) {
            if (!live[q]) continue;
            const int d = dd[q];
            T val;
            if (inb[q]) {
                val = sc[q];
                if (begin) begin_fold<Sm>(c, d, val, bsc);
            } else {
                val = d == 0 ? base0 : ZERO;
            }
            Sm::st(dst + d, val);
        }
    }
}

// IL chain over the band by one warp, KC cells per lane in registers.
template <class Sm, int KC>
__device__ __forceinline__ void il_relax(const Ctx &c, const Col &C, int v, const St &s, const uint32_t *const *kp,
                                         const typename Sm::T *ts, bool endsc, typename Sm::T es, bool begin,
                                         typename Sm::T bsc, uint32_t *dst, int dn, int dx, int kk) {
    typedef typename Sm::T T;
    const T ZERO = Sm::zero();
    const T t0 = ts[0];
    T cv[KC], ev[KC], xv[KC];
    const int dbeg = dn + c.lane * kk;
    const bool has = dbeg <= dx;
#pragma unroll
    for (int q = 0; q < KC; q++) {
        const int d = dbeg + q;
        cv[q] = ZERO;
        ev[q] = ZERO;
        xv[q] = ZERO;
        if (q < kk && d <= dx) {
            T terms[6];
            terms[0] = ZERO;
#pragma unroll
            for (int yo = 1; yo < 6; yo++)
                if (yo < s.cnum) terms[yo] = Sm::add(Sm::ld(kp[yo] + d), ts[yo]);
            const T init = endsc ? Sm::add(Sm::ld(c.el + d - 1), es) : ZERO;
            cv[q] = reduce_c_noself<Sm>(s.cnum, terms, init, c.tbl, c.nz);
            ev[q] = esc1<Sm>(c, v, s.escoff, c.ring[(C.j - d + 1) & c.rmask]);
        }
    }
    // the cell below the band is an unwritten emitter cell: zero
    T xin = ZERO, xin_prev = ZERO;
    for (int it = 0; it < 34; it++) {
        T x = xin;
#pragma unroll
        for (int q = 0; q < KC; q++) {
            if (q < kk && dbeg + q <= dx) {
                x = Sm::add(Sm::comb(cv[q], Sm::add(x, t0), c.tbl, c.nz), ev[q]);
                xv[q] = x;
            }
        }
        const T xlast = has ? x : ZERO;
        const bool same = !has || Sm::u(xin) == Sm::u(xin_prev);
        if (it > 0 && __all_sync(FULL, same)) break;
        xin_prev = xin;
        const T up = __shfl_up_sync(FULL, xlast, 1);
        xin = c.lane == 0 ? ZERO : up;
    }
#pragma unroll
    for (int q = 0; q < KC; q++) {
        const int d = dbeg + q;
        if (q < kk && d <= dx) {
            Sm::st(dst + d, xv[q]);
            if (begin) begin_fold<Sm>(c, d, xv[q], bsc);
        }
    }
}

template <class Sm>
__device__ __forceinline__ void do_il(const Ctx &c, const Col &C, int v, const St &s, int par, uint32_t *dst) {
    typedef typename Sm::T T;
    const T ZERO = Sm::zero();
    const uint32_t *kp[6];
    T ts[6];
#pragma unroll
    for (int yo = 0; yo < 6; yo++) {
        kp[yo] = c.buf;
        ts[yo] = ZERO;
        if (yo < s.cnum) {
            kp[yo] = kid_base(c, c.kid[v * 6 + yo], par, 0) - 1;  // IL reads no previous column
            ts[yo] = Sm::ld(c.tsc + v * 6 + yo);
        }
    }
    const bool endsc = s.flags & SF_ENDSC;
    const T es = endsc ? Sm::ld(c.endsc + v) : ZERO;
    const bool begin = s.flags & SF_BEGIN;
    const T bsc = begin ? Sm::ld(c.bsv + v) : ZERO;
    const int dn = s.dn, dx = min(C.jrow, s.dxcap);
    const int n = dx - dn + 1;
    if (n > 0) {
        const int kk = (n + 31) >> 5;
#define IL_CASE(KC) \
    case KC: il_relax<Sm, KC>(c, C, v, s, kp, ts, endsc, es, begin, bsc, dst, dn, dx, kk); break;
        switch (kk) {
            IL_CASE(1)
            IL_CASE(2)
            IL_CASE(3)
            IL_CASE(4)
            IL_CASE(5)
            IL_CASE(6)
            IL_CASE(7)
            default: il_relax<Sm, 8>(c, C, v, s, kp, ts, endsc, es, begin, bsc, dst, dn, dx, kk);
        }
#undef IL_CASE
    }
    const T base0 = Sm::ld(c.init0 + v);
    for (int d = s.lo + c.lane; d <= s.hi; d += 32)
        if (d < dn || d > dx) Sm::st(dst + d, d == 0 ? base0 : ZERO);
}

// Bifurcation: cell d = init (+) over k ascending of BEGL(j-k, d-k) +
// BEGR(j, k).  The 32 cells of a round step through a common k so that each
// step reads one contiguous piece of a ring column.
template <class Sm>
__device__ __forceinline__ void do_bif(const Ctx &c, const Col &C, int v, const St &s, int par, int bi) {
    typedef typename Sm::T T;
    const T ZERO = Sm::zero();
    const int4 bq = c.bifs[bi];
    const int kdn_y = (int16_t)(bq.x & 0xffff), kdx_y = (int16_t)((uint32_t)bq.x >> 16);
    const int kdn_w = (int16_t)(bq.y & 0xffff), kdx_w = (int16_t)((uint32_t)bq.y >> 16);
    const uint32_t *ring = c.rings + (size_t)bi * c.RW * c.S;
    const uint32_t *begr = c.begr + bi * c.S;
    uint32_t *dst = c.buf + (par * SW_SLOTS + s.slot) * c.S;
    const bool endsc = s.flags & SF_ENDSC;
    const T es = endsc ? Sm::ld(c.endsc + v) : ZERO;
    const bool begin = s.flags & SF_BEGIN;
    const T bsc = begin ? Sm::ld(c.bsv + v) : ZERO;
    const T base0 = Sm::ld(c.init0 + v);
    const int dx = min(C.jrow, s.dxcap);
    for (int d0 = s.lo; d0 <= s.hi; d0 += 32) {
        const int d = d0 + c.lane;
        const bool live = d <= s.hi;
        const bool inb = live && d >= s.dn && d <= dx;
        const int kmin = max(0, max(kdn_y, d - kdx_w));
        const int kmax = min(kdx_y, d - kdn_w);
        const bool act = inb && kmin <= kmax;
        const int K0 = __reduce_min_sync(FULL, act ? kmin : INT_MAX);
        const int K1 = __reduce_max_sync(FULL, act ? kmax : INT_MIN);
        T sc = (inb && endsc) ? Sm::add(Sm::ld(c.el + d), es) : ZERO;
        if (K0 <= K1) {
            // eight steps at a time: the ring loads of a batch are issued
            // before its folds, which stay in ascending k
            constexpr int KB = 8;
            int col = C.jm - K0;
            if (col < 0) col += c.RW;
            for (int k0 = K0; k0 <= K1; k0 += KB) {
                T lv[KB], rv[KB];
#pragma unroll
                for (int u = 0; u < KB; u++) {
                    const int k = k0 + u;
                    int cc = col - u;
                    if (cc < 0) cc += c.RW;
                    const bool on = act && k >= kmin && k <= kmax;
                    lv[u] = on ? Sm::ld(ring + (size_t)cc * c.S + d - k) : ZERO;
                    rv[u] = on ? Sm::ld(begr + k) : ZERO;
                }
#pragma unroll
                for (int u = 0; u < KB; u++) {
                    const int k = k0 + u;
                    if (act && k >= kmin && k <= kmax) sc = Sm::comb(sc, Sm::add(lv[u], rv[u]), c.tbl, c.nz);
                }
                col -= KB;
                if (col < 0) col += c.RW;
            }
        }
        if (live) {
            const T val = inb ? sc : (d == 0 ? base0 : ZERO);
            Sm::st(dst + d, val);
            if (begin && inb) begin_fold<Sm>(c, d, val, bsc);
        }
    }
}

// ROOT_S: children in plain order, then local begins (MAX), then every
// reportable cell of a reported column goes to the candidate buffer.
template <class Sm>
__device__ __forceinline__ void do_root(const Ctx &c, const Col &C, const St &s, int par) {
    typedef typename Sm::T T;
    const T ZERO = Sm::zero();
    const uint32_t *kp[6];
    T ts[6];
#pragma unroll
    for (int yo = 0; yo < 6; yo++) {
        kp[yo] = c.buf;
        ts[yo] = ZERO;
        if (yo < s.cnum) {
            kp[yo] = kid_base(c, c.kid[yo], par, 0);  // ROOT_S reads the current column
            ts[yo] = Sm::ld(c.tsc + yo);
        }
    }
    const SweepParams &p = *c.p;
    const int dx = min(C.jrow, s.dxcap);
    for (int d0 = s.dn; d0 <= dx; d0 += 32) {
        const int d = d0 + c.lane;
        bool hit = false;
        T a = ZERO;
        if (d <= dx) {
            a = Sm::comb(ZERO, Sm::add(Sm::ld(kp[0] + d), ts[0]), c.tbl, c.nz);
#pragma unroll
            for (int yo = 1; yo < 6; yo++)
                if (yo < s.cnum) a = Sm::comb(a, Sm::add(Sm::ld(kp[yo] + d), ts[yo]), c.tbl, c.nz);
            if (p.local) {
                const T cand = Sm::ld(c.bmax + d);
                Sm::st(c.bmax + d, ZERO);
                if (a < cand) a = cand;
            }
            if (C.j >= C.jreport) {
                const float sc = Sm::bits(a);
                hit = sc >= p.cutoff && sc > IMPOSSIBLE_D + 1.0f;
            }
        }
        const unsigned m = __ballot_sync(FULL, hit);
        if (m) {
            const int leader = __ffs(m) - 1;
            int base = 0;
            if (c.lane == leader) base = atomicAdd(p.cand_count, __popc(m));
            base = __shfl_sync(FULL, base, leader);
            if (hit) {
                const int pos = base + __popc(m & ((1u << c.lane) - 1));
                if (pos < p.cand_cap) {
                    Cand cd;
                    cd.item = p.item_base + C.item;
                    cd.j = C.j;
                    cd.d = d;
                    cd.raw = Sm::u(a);
                    p.cands[pos] = cd;
                }
            }
        }
    }
}

// Previous-column values node n reads: deck slots -> previous-column buffer
// pb, with cp.async (completion awaited before node n runs); in the first
// column of a work item the reference's initial deck fill instead.
template <class Sm>
__device__ __forceinline__ void prefetch(const Ctx &c, const Col &C, int n, int pb) {
    const int4 nq = c.nodes[n];
    const int nio = (nq.x >> 16) & 0xff, io0 = (int16_t)((uint32_t)nq.y >> 16);
    const uint32_t zero = Sm::u(Sm::zero());
    for (int e = 0; e < nio; e++) {
        const int4 q = c.io[io0 + e];
        const int y = (int16_t)(q.x & 0xffff), pslot = (q.x >> 16) & 0xff;
        const int lo = (int16_t)(q.y & 0xffff), hi = (int16_t)((uint32_t)q.y >> 16);
        uint32_t *dstb = c.buf + (12 + pb * SW_SLOTS + pslot) * c.S;
        if (C.first) {
            const uint32_t b0 = c.init0[y];
            for (int d = lo + c.lane; d <= hi; d += 32) dstb[d] = d == 0 ? b0 : zero;
        } else {
            const uint32_t *g = c.deck + q.z;
            for (int d = lo + c.lane; d <= hi; d += 32) cp_async4(dstb + d, g + d);
        }
    }
    cp_async_commit();
}

template <class Sm>
__device__ __forceinline__ void do_column(const Ctx &c, const Col &C) {
    const SweepParams &p = *c.p;
    const int S = c.S;
    int pb = 0;
    prefetch<Sm>(c, C, p.nnodes - 1, pb);
    for (int n = p.nnodes - 1; n >= 0; n--) {
        const int4 nq = c.nodes[n];
        const int nst = (nq.x >> 8) & 0xff, nio = (nq.x >> 16) & 0xff;
        const int aux = ((uint32_t)nq.x >> 24) & 0xff;
        const int v0 = (int16_t)(nq.y & 0xffff), io0 = (int16_t)((uint32_t)nq.y >> 16);
        const int par = n & 1;
        // this node's previous-column values have arrived; fetch the next
        // node's while this one computes
        cp_async_wait_all();
        __syncwarp();
        if (n > 0) prefetch<Sm>(c, C, n - 1, pb ^ 1);
        for (int v = v0 + nst - 1; v >= v0; v--) {
            const St s = unpack(c.st[v]);
            if (s.type == E_ST_D) {
                uint32_t *dst = c.buf + (par * SW_SLOTS + s.slot) * S;
                const uint32_t b0 = c.init0[v];
                const uint32_t zero = Sm::u(Sm::zero());
                for (int d = s.lo + c.lane; d <= s.hi; d += 32) dst[d] = d == 0 ? b0 : zero;
            } else if (s.type == B_ST_D) {
                do_bif<Sm>(c, C, v, s, par, aux);
            } else if (s.flags & SWF_ROOT) {
                do_root<Sm>(c, C, s, par);
            } else if (s.type == IL_ST_D) {
                do_il<Sm>(c, C, v, s, par, c.buf + (par * SW_SLOTS + s.slot) * S);
            } else {
                uint32_t *dst;
                if (s.flags & SWF_BEGL)
                    dst = c.rings + (size_t)aux * c.RW * S + (size_t)C.jm * S;
                else if (s.flags & SWF_BEGR)
                    dst = c.begr + aux * S;
                else
                    dst = c.buf + (par * SW_SLOTS + s.slot) * S;
                do_plain<Sm>(c, C, v, s, par, pb, dst);
            }
            __syncwarp();
        }
        // current values of those states to the deck, for the next column
        for (int e = 0; e < nio; e++) {
            const int4 q = c.io[io0 + e];
            const int cur = ((uint32_t)q.x >> 24) & 0xff;
            const int lo = (int16_t)(q.y & 0xffff), hi = (int16_t)((uint32_t)q.y >> 16);
            const uint32_t *src = cur < 8 ? c.buf + (par * SW_SLOTS + cur) * S
                                          : c.buf + ((par ^ 1) * SW_SLOTS + cur - 8) * S;
            uint32_t *g = c.deck + q.z;
            for (int d = lo + c.lane; d <= hi; d += 32) g[d] = src[d];
        }
        __syncwarp();
        pb ^= 1;
    }
}

template <bool INS>
__global__ void __launch_bounds__(SW_MAX_WARPS * 32, 1) sweep_kernel(SweepParams p) {
    typedef typename SemSel<INS>::type Sm;
    extern __shared__ __align__(16) uint32_t smem[];
    const SwLayout &ly = p.lay;
    const int tid = threadIdx.x, bs = blockDim.x;
    {
        auto copy32 = [&](int dst, const void *src, int n) {
            const uint32_t *g = reinterpret_cast<const uint32_t *>(src);
            for (int x = tid; x < n; x += bs) smem[dst + x] = __ldg(g + x);
        };
        copy32(ly.st, p.st, p.M * 4);
        copy32(ly.kid, p.kid, (p.M * 6 + 3) / 4);
        copy32(ly.tsc, p.tsc, p.M * 6);
        copy32(ly.endsc, p.endsc, p.M);
        copy32(ly.init0, p.init0, p.M);
        copy32(ly.bsv, p.bsv, p.M);
        copy32(ly.escc, p.esc_c, p.n_esc_c);
        copy32(ly.el, p.el_sca, p.W + 1);
        if (INS) {
            copy32(ly.tbl, p.ilog, p.ilog_nz / 2);
            // the last (odd) entry, then the zero entry at nz
            if (tid == 0) {
                uint16_t *t16 = reinterpret_cast<uint16_t *>(smem + ly.tbl);
                if (p.ilog_nz & 1) t16[p.ilog_nz - 1] = p.ilog[p.ilog_nz - 1];
                t16[p.ilog_nz] = 0;
            }
        }
        copy32(ly.nodes, p.nodes, p.nnodes * 4);
        copy32(ly.io, p.io, p.nio * 4);
        copy32(ly.bifs, p.bifs, p.nbif * 4);
    }
    const int lane = tid & 31, warp = tid >> 5;
    Ctx c;
    c.p = &p;
    c.st = reinterpret_cast<const int4 *>(smem + ly.st);
    c.kid = reinterpret_cast<const uint8_t *>(smem + ly.kid);
    c.tsc = smem + ly.tsc;
    c.endsc = smem + ly.endsc;
    c.init0 = smem + ly.init0;
    c.bsv = smem + ly.bsv;
    c.escc = smem + ly.escc;
    c.el = smem + ly.el;
    c.tbl = reinterpret_cast<const uint16_t *>(smem + ly.tbl);
    c.nz = p.ilog_nz;
    c.nodes = reinterpret_cast<const int4 *>(smem + ly.nodes);
    c.io = reinterpret_cast<const int4 *>(smem + ly.io);
    c.bifs = reinterpret_cast<const int4 *>(smem + ly.bifs);
    c.S = p.S;
    c.RW = p.RW;
    c.lane = lane;
    uint32_t *wsm = smem + ly.warp0 + (size_t)warp * ly.wwords;
    c.buf = wsm;
    c.begr = wsm + 24 * p.S;
    c.bmax = c.begr + p.nbif * p.S;
    c.ring = reinterpret_cast<uint8_t *>(c.bmax + p.S);
    c.rmask = ly.ring_len - 1;
    uint32_t *gw = p.gmem + ((size_t)blockIdx.x * p.warps + warp) * (size_t)p.gstride;
    c.deck = gw;
    c.rings = gw + p.deck_words;
    // per-warp state: local-begin row and residue ring start clear
    for (int d = lane; d < p.S; d += 32) Sm::st(c.bmax + d, Sm::zero());
    for (int x = lane; x < ly.ring_len; x += 32) c.ring[x] = 0;
    __syncthreads();
    {
        const St r = unpack(c.st[0]);
        c.rdn = r.dn;
        c.rdx = r.dxcap;
    }

    for (;;) {
        int it = 0;
        if (lane == 0) it = atomicAdd(p.next_item, 1);
        it = __shfl_sync(FULL, it, 0);
        if (it >= p.nitems) break;
        const WorkItem wi = p.items[it];
        // d = 0 cells of every BEGL ring column hold the BEGL_S base value
        for (int b = 0; b < p.nbif; b++) {
            const int4 bq = c.bifs[b];
            const int w = (int16_t)(bq.z & 0xffff);
            const St sw = unpack(c.st[w]);
            if (sw.lo > 0) continue;
            const uint32_t b0 = c.init0[w];
            uint32_t *ring = c.rings + (size_t)b * p.RW * p.S;
            for (int col = lane; col < p.RW; col += 32) ring[(size_t)col * p.S] = b0;
        }
        __syncwarp();
        Col C;
        C.item = it;
        C.jreport = wi.jreport;
        int jm = wi.jstart % p.RW;
        for (int j = wi.jstart; j <= wi.jend; j++) {
            if (((j - wi.jstart) & 31) == 0) {
                __syncwarp();
                const int x = j + lane;
                if (x <= wi.jend) {
                    const int cc = __ldg(p.dsq + wi.dsq_off + x);
                    c.ring[x & c.rmask] = (uint8_t)(cc > 17 ? 17 : cc);
                }
                __syncwarp();
            }
            C.j = j;
            C.jrow = min(j - wi.jstart + 1, p.W);
            C.jm = jm;
            C.first = j == wi.jstart;
            C.resj = c.ring[j & c.rmask];
            do_column<Sm>(c, C);
            jm = jm + 1 == p.RW ? 0 : jm + 1;
        }
    }
}

}  // namespace swdev

SwLayout sweep_layout(const SweepParams &p, int warps) {
    SwLayout L{};
    int64_t w = 0;
    auto take = [&](int64_t n) {
        int64_t o = w;
        w += (n + 3) & ~(int64_t)3;  // 16-byte alignment
        return (int)o;
    };
    L.st = take((int64_t)p.M * 4);
    L.kid = take(((int64_t)p.M * 6 + 3) / 4);
    L.tsc = take((int64_t)p.M * 6);
    L.endsc = take(p.M);
    L.init0 = take(p.M);
    L.bsv = take(p.M);
    L.escc = take(p.n_esc_c);
    L.el = take(p.W + 1);
    L.tbl = take(p.inside ? p.ilog_nz / 2 + 1 : 0);
    L.nodes = take((int64_t)p.nnodes * 4);
    L.io = take((int64_t)p.nio * 4);
    L.bifs = take((int64_t)p.nbif * 4);
    int r = 32;
    while (r < p.W + 33) r <<= 1;
    L.ring_len = r;
    L.wwords = (int)(((int64_t)(24 + p.nbif + 1) * p.S + r / 4 + 3) & ~(int64_t)3);
    L.warp0 = (int)w;
    w += (int64_t)warps * L.wwords;
    L.words = w;
    return L;
}

template <bool INS>
static int occ_t(const SweepParams &p, int threads) {
    int n = 0;
    auto kern = swdev::sweep_kernel<INS>;
    size_t smem = (size_t)p.lay.words * 4;
    if (cmx::allow_max_dynamic_smem(kern) != cudaSuccess) return 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kern, threads, smem) != cudaSuccess) return 0;
    return n;
}

int sweep_occupancy(const SweepParams &p, int threads) {
    return p.inside ? occ_t<true>(p, threads) : occ_t<false>(p, threads);
}

template <bool INS>
static cudaError_t launch_t(const SweepParams &p, int ctas, cudaStream_t s) {
    auto kern = swdev::sweep_kernel<INS>;
    size_t smem = (size_t)p.lay.words * 4;
    cudaError_t e = cmx::allow_max_dynamic_smem(kern);
    if (e != cudaSuccess) return e;
    kern<<<ctas, p.warps * 32, smem, s>>>(p);
    return cudaGetLastError();
}

cudaError_t sweep_launch(const SweepParams &p, int ctas, cudaStream_t s) {
    return p.inside ? launch_t<true>(p, ctas, s) : launch_t<false>(p, ctas, s);
}

}  // namespace cmx
