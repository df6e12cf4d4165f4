// QDB-banded CYK / Inside window scanner for sm_100a.
//
// Work decomposition.  A window is cut into work items: a piece of the
// window plus W-1 warm-up columns.  A cell (j,d) depends only on residues
// j-d+1..j, so a piece started W-1 columns early reproduces the reference's
// cells bit for bit (src/cm_nohmm.rs:549-763 computes them with
// jrow = min(j-i0+1, W)).  Items sit in a cost-ordered device queue; each
// persistent CTA runs `lanes` items side by side (one deck per lane, one copy
// of the model metadata), refilling a lane from the queue when its item ends.
//
// Per column the CTA walks the plan's levels for every lane at once:
//   level 0   every right emitter (MP, MR, IR).  They read only column j-1
//             (jp_y = prv, src/cm_nohmm.rs:575), so all of them are
//             independent and run in one phase;
//   level l   states whose same-column children sit in levels < l;
//   root      ROOT_S transitions, local begins (MAX in both semirings,
//             src/cm_nohmm.rs:700-746) and candidate emission.
// Warps take (lane, state, 32 cells) units; lanes of a warp are consecutive
// d.  Cells are evaluated in the reference's operand order (reduce_c_order,
// src/cm_nohmm.rs:187-242, for emitters, S and D states; natural child order
// for BEGL_S, :601-611; ascending k for bifurcations), so integer ILogsum
// results are bit-identical; f32 adds use __fadd_rn (no contraction).
//
// IL states read their own cell d-1 (self loop, src/cm_nohmm.rs:622-649), a
// serial chain in d.  One warp resolves it by blocked fixed-point iteration:
// lane l owns a block of consecutive d, walks it serially from an incoming
// value and passes its last value to lane l+1; the warp repeats until no
// incoming value changes.  When nothing changes the values satisfy the
// serial recurrence everywhere, so they are the serial result; after r rounds
// lanes 0..r are exact, so 33 rounds always suffice.
//
// Decks: right emitters keep two column slots (j & 1), BEGL_S states a ring
// of W+1 columns, every other state one slot that level 0 of column j reads
// (as column j-1) before levels >= 1 overwrite it.  Decks live in shared
// memory when they fit, else in a per-(CTA, lane) region of global memory.
// Metadata, score tables (canonical residues), the ILogsum table and a
// residue ring per lane always live in shared memory.
#include <cuda_runtime.h>
#include <cstdint>

#include "devbuf.h"
#include "qdb_kernel.h"
#include "semiring.cuh"

namespace cmx {
namespace dev {

struct SInfo {  // unpacked StateDev
    int dn, dxcap, cnum, type, flags, sd, escoff, span;
};

__device__ __forceinline__ SInfo unpack(int4 q) {
    SInfo s;
    s.dn = (int16_t)(q.x & 0xffff);
    s.dxcap = (int16_t)((uint32_t)q.x >> 16);
    s.cnum = q.y & 0xff;
    s.type = (q.y >> 8) & 0xff;
    s.flags = (q.y >> 16) & 0xff;
    s.sd = ((uint32_t)q.y >> 24) & 0xff;
    s.escoff = q.z;
    s.span = q.w;
    return s;
}

// Shared-memory views of the model and the per-lane state.
struct Smem {
    const uint32_t *el;
    const uint16_t *tbl;
    const int4 *info;
    const int32_t *wb, *cb;
    const uint32_t *tsc, *endsc, *escc, *beginsc;
    const uint32_t *bsv;  // [M] begin score per state (fused begins)
    int32_t *bmax;        // [lanes][bstride] ROOT-row begin maxima (fused begins)
    uint32_t *prow;       // [lanes][bstride] ROOT-row raw values (report pre-filter)
    int bstride;
    const int32_t *lvl;
    const int4 *begin;
    const int2 *chunks;
    uint8_t *ring;
    int32_t *lane;  // [MAX_LANES][8]
};

// Per-lane view of one column.
struct Lane {
    uint32_t *deck;
    const uint8_t *ring;  // residue at position x: ring[x & rmask]
    int j, par, jm, jrow;
    int l;                // lane (work item slot) index
};

struct K {
    const ScanParams *p;
    Smem s;
    int nz;
    int rmask;
    // scalars the per-cell code reads, held in registers
    const uint32_t *esc_g;  // full emission rows [M][324] (IUPAC codes)
    int fuse_begin, begin_key, root_dn, root_dxcap, W1;
};

// Emission score of a single residue / a pair; canonical residues come from
// shared memory, IUPAC codes from the full 18 / 18x18 rows in global memory.
template <class S>
__device__ __forceinline__ typename S::T esc1(const K &k, int v, int escoff, int c) {
    if (c < 4) return S::ld(k.s.escc + escoff + c);
    return S::ldg(k.esc_g + v * 324 + c);
}
template <class S>
__device__ __forceinline__ typename S::T esc2(const K &k, int v, int escoff, int a, int b) {
    if ((a | b) < 4) return S::ld(k.s.escc + escoff + a * 4 + b);
    return S::ldg(k.esc_g + v * 324 + a * 18 + b);
}

// Child terms of cell d: deck[cb[v][yo][par] + d] + tsc[v][yo].  The padded
// deck layout makes every read a plain load (no band test).
template <class S>
__device__ __forceinline__ void child_terms(const K &k, int v, int cnum, const uint32_t *deck, int par, int d,
                                            typename S::T *terms, int first) {
    const int32_t *cb = k.s.cb + v * 12 + par;
    const uint32_t *tsc = k.s.tsc + v * 6;
#pragma unroll
    for (int yo = 0; yo < 6; yo++)
        if (yo >= first && yo < cnum) terms[yo] = S::add(S::ld(deck + cb[2 * yo] + d), S::ld(tsc + yo));
}

template <class S>
__device__ __forceinline__ typename S::T init_sc(const K &k, const SInfo &sv, int v, int idx) {
    if (sv.flags & SF_ENDSC) return S::add(S::ld(k.s.el + idx), S::ld(k.s.endsc + v));
    return S::zero();
}

__device__ __forceinline__ int resid(const Lane &L, int x, int rmask) { return L.ring[x & rmask]; }

// Value of cell d of an ordinary state (not B, not IL) with CN children,
// before the store.  CN is a compile-time constant, so the child loop and the
// reduce_c_order switch unroll to exactly the state's children.
template <class S, int CN>
__device__ __forceinline__ typename S::T cell_value(const K &k, const Lane &L, int v, const SInfo &sv, int d) {
    typedef typename S::T T;
    const int t = sv.type;
    T terms[6];
    child_terms<S>(k, v, CN, L.deck, L.par, d, terms, 0);
    const int idx = d - sv.sd;
    T sc;
    if (sv.flags & SF_BEGL) {
        // BEGL_S folds its children in natural order (src/cm_nohmm.rs:601-611)
        sc = init_sc<S>(k, sv, v, idx);
#pragma unroll
        for (int yo = 0; yo < CN; yo++) sc = S::comb(sc, terms[yo], k.s.tbl, k.nz);
    } else {
        sc = reduce_c<S>(CN, terms, init_sc<S>(k, sv, v, idx), k.s.tbl, k.nz);
    }
    if (t == 2 || t == 4) {  // ML, IL: residue i = j-d+1
        sc = S::add(sc, esc1<S>(k, v, sv.escoff, resid(L, L.j - d + 1, k.rmask)));
    } else if (t == 3 || t == 5) {  // MR, IR: residue j
        sc = S::add(sc, esc1<S>(k, v, sv.escoff, resid(L, L.j, k.rmask)));
    } else if (t == 1) {  // MP
        sc = S::add(sc, esc2<S>(k, v, sv.escoff, resid(L, L.j - d + 1, k.rmask), resid(L, L.j, k.rmask)));
    }
    return sc;
}

// Local-begin comparison: `a < cand` on the raw values (src/cm_nohmm.rs:
// 720-742), or, for cmcalibrate's scan (src/cm_calibrate.rs:720-745), on
// their bit scores, where -INFTY (IMPOSSIBLE) sits below every other integer.
template <class S>
__device__ __forceinline__ bool begin_less(int key, typename S::T a, typename S::T cand) {
    if (S::ORDERED && key) {
        const int32_t ka = (int32_t)S::u(a) == -INFTY_D ? INT32_MIN : (int32_t)S::u(a);
        const int32_t kc = (int32_t)S::u(cand) == -INFTY_D ? INT32_MIN : (int32_t)S::u(cand);
        return ka < kc;
    }
    return a < cand;
}

// Fused local begins (integer Inside): ROOT cell d takes the maximum of
// cell(v, d) + beginsc[v] over the begin states v, and a maximum needs no
// order, so each begin state posts its cells as it computes them.
template <class S>
__device__ __forceinline__ void post_begin(const K &k, const Lane &L, const SInfo &sv, int v, int d,
                                           typename S::T x) {
    if (S::ORDERED && k.fuse_begin && (sv.flags & SF_BEGIN) && d >= k.root_dn && d <= min(L.jrow, k.root_dxcap)) {
        int32_t c = (int32_t)((uint32_t)S::u(x) + k.s.bsv[v]);
        if (k.begin_key && c == -INFTY_D) c = INT32_MIN;
        atomicMax(k.s.bmax + L.l * k.s.bstride + d, c);
    }
}

// One warp-wide chunk of an ordinary state (not B, not IL): 64 cells, two per
// lane (d0+lane and d0+32+lane).  Both values are computed before either is
// stored, so the two dependency chains overlap.
template <class S, int CN>
__device__ __forceinline__ void do_chunk_c(const K &k, const Lane &L, int v, const SInfo &sv, int d0, int lane) {
    typedef typename S::T T;
    const int dx = min(L.jrow, sv.dxcap);
    const int da = d0 + lane, db = da + 32;
    if (da > dx) return;
    const bool has_b = db <= dx;
    T va = cell_value<S, CN>(k, L, v, sv, da);
    T vb = has_b ? cell_value<S, CN>(k, L, v, sv, db) : va;
    const int wbase = (sv.flags & SF_BEGL) ? k.s.wb[v * 2] + L.jm * sv.span : k.s.wb[v * 2 + L.par];
    S::st(L.deck + wbase + da, va);
    if (has_b) S::st(L.deck + wbase + db, vb);
    post_begin<S>(k, L, sv, v, da, va);
    if (has_b) post_begin<S>(k, L, sv, v, db, vb);
}

// cnum is 1..6 for every non-B, non-E state of a CM
template <class S>
__device__ __forceinline__ void do_chunk(const K &k, const Lane &L, int v, const SInfo &sv, int d0, int lane) {
    switch (sv.cnum) {
    case 1: do_chunk_c<S, 1>(k, L, v, sv, d0, lane); break;
    case 2: do_chunk_c<S, 2>(k, L, v, sv, d0, lane); break;
    case 3: do_chunk_c<S, 3>(k, L, v, sv, d0, lane); break;
    case 4: do_chunk_c<S, 4>(k, L, v, sv, d0, lane); break;
    case 5: do_chunk_c<S, 5>(k, L, v, sv, d0, lane); break;
    default: do_chunk_c<S, 6>(k, L, v, sv, d0, lane); break;
    }
}

// Bifurcation cell: alpha[v][d] = init (+) over k ascending of
// BEGL(j-k, d-k) + BEGR(j, k) (src/cm_nohmm.rs:578-600).
template <class S>
__device__ __forceinline__ typename S::T bif_value(const K &k, const Lane &L, int v, const SInfo &sv, int d) {
    typedef typename S::T T;
    const int32_t *c = k.s.cb + v * 12;
    const int begl = c[0], begr = c[2], kdn_y = c[4], kdx_y = c[5], kdn_w = c[6], kdx_w = c[7], span_w = c[8];
    const int kmin = max(0, max(kdn_y, d - kdx_w));
    const int kmax = min(kdx_y, d - kdn_w);
    T sc = init_sc<S>(k, sv, v, d);
    const int W1 = k.W1;
    int col = L.jm - kmin;
    if (col < 0) col += W1;
    const uint32_t *left = L.deck + begl + d;
    const uint32_t *right = L.deck + begr;
    for (int kk = kmin; kk <= kmax; kk++) {
        T lv = S::ld(left + col * span_w - kk);
        T rv = S::ld(right + kk);
        sc = S::comb(sc, S::add(lv, rv), k.s.tbl, k.nz);
        col = col == 0 ? W1 - 1 : col - 1;
    }
    return sc;
}

// Bifurcation chunk: 64 cells, two per lane, computed before the stores.
template <class S>
__device__ __forceinline__ void do_bif_chunk(const K &k, const Lane &L, int v, const SInfo &sv, int d0, int lane) {
    typedef typename S::T T;
    const int dx = min(L.jrow, sv.dxcap);
    const int da = d0 + lane, db = da + 32;
    if (da > dx) return;
    const bool has_b = db <= dx;
    T va = bif_value<S>(k, L, v, sv, da);
    T vb = has_b ? bif_value<S>(k, L, v, sv, db) : va;
    const int wb = k.s.wb[v * 2 + L.par];
    S::st(L.deck + wb + da, va);
    if (has_b) S::st(L.deck + wb + db, vb);
    post_begin<S>(k, L, sv, v, da, va);
    if (has_b) post_begin<S>(k, L, sv, v, db, vb);
}

// IL relaxation with up to KC cells per lane held in registers.
template <class S, int KC>
__device__ __forceinline__ void il_relax(const K &k, const Lane &L, int v, const SInfo &sv, int dn, int dx, int kk,
                                         int lane) {
    typedef typename S::T T;
    const T t0 = S::ld(k.s.tsc + v * 6);
    uint32_t *dst = L.deck + k.s.wb[v * 2];  // IL is single-slot
    T cv[KC], ev[KC], xv[KC];
    const int dbeg = dn + lane * kk;
    const bool has = dbeg <= dx;
#pragma unroll
    for (int q = 0; q < KC; q++) {
        int d = dbeg + q;
        cv[q] = S::zero();
        ev[q] = S::zero();
        xv[q] = S::zero();
        if (q < kk && d <= dx) {
            T terms[6];
            child_terms<S>(k, v, sv.cnum, L.deck, L.par, d, terms, 1);
            cv[q] = reduce_c_noself<S>(sv.cnum, terms, init_sc<S>(k, sv, v, d - 1), k.s.tbl, k.nz);
            ev[q] = esc1<S>(k, v, sv.escoff, resid(L, L.j - d + 1, k.rmask));
        }
    }
    // x at d = dn-1 is an unwritten cell of the emitter: zero.
    T xin = S::zero(), xin_prev = S::zero();
    for (int it = 0; it < 34; it++) {
        T x = xin;
#pragma unroll
        for (int q = 0; q < KC; q++) {
            if (q < kk && dbeg + q <= dx) {
                x = S::add(S::comb(cv[q], S::add(x, t0), k.s.tbl, k.nz), ev[q]);
                xv[q] = x;
            }
        }
        // a lane without cells passes nothing on
        T xlast = has ? x : S::zero();
        bool same = !has || S::u(xin) == S::u(xin_prev);
        if (it > 0 && __all_sync(0xffffffffu, same)) break;
        xin_prev = xin;
        T up = __shfl_up_sync(0xffffffffu, xlast, 1);
        xin = lane == 0 ? S::zero() : up;
    }
#pragma unroll
    for (int q = 0; q < KC; q++) {
        int d = dbeg + q;
        if (q < kk && d <= dx) S::st(dst + d, xv[q]);
    }
}

// IL state: whole band by one warp (see the file comment).
template <class S>
__device__ __forceinline__ void do_il(const K &k, const Lane &L, int v, const SInfo &sv, int lane) {
    typedef typename S::T T;
    const int dn = sv.dn;
    const int dx = min(L.jrow, sv.dxcap);
    const int n = dx - dn + 1;
    if (n <= 0) return;
    const int kk = (n + 31) >> 5;
    if (kk == 1) {
        il_relax<S, 1>(k, L, v, sv, dn, dx, kk, lane);
    } else if (kk == 2) {
        il_relax<S, 2>(k, L, v, sv, dn, dx, kk, lane);
    } else if (kk <= 4) {
        il_relax<S, 4>(k, L, v, sv, dn, dx, kk, lane);
    } else if (kk <= IL_KMAX) {
        il_relax<S, IL_KMAX>(k, L, v, sv, dn, dx, kk, lane);
    } else {
        // wide band: c in parallel into the deck, then one lane walks d
        const T t0 = S::ld(k.s.tsc + v * 6);
        uint32_t *dst = L.deck + k.s.wb[v * 2];
        for (int d = dn + lane; d <= dx; d += 32) {
            T terms[6];
            child_terms<S>(k, v, sv.cnum, L.deck, L.par, d, terms, 1);
            S::st(dst + d, reduce_c_noself<S>(sv.cnum, terms, init_sc<S>(k, sv, v, d - 1), k.s.tbl, k.nz));
        }
        __syncwarp();
        if (lane == 0) {
            T x = S::zero();
            for (int d = dn; d <= dx; d++) {
                T e = esc1<S>(k, v, sv.escoff, resid(L, L.j - d + 1, k.rmask));
                x = S::add(S::comb(S::ld(dst + d), S::add(x, t0), k.s.tbl, k.nz), e);
                S::st(dst + d, x);
            }
        }
        __syncwarp();
    }
}

// lane-state fields in shared memory
enum { LS_ITEM = 0, LS_JB, LS_JSTART, LS_JEND, LS_JREPORT, LS_OFFLO, LS_OFFHI, LS_JM };
constexpr int LS_W = 8;

// Appends the cells of the warp's lanes with hit set to the candidate buffer
// (one atomic per warp); entries past cand_cap are counted, not written.
__device__ __forceinline__ void emit_cand(const ScanParams &p, int wl, bool hit, int item, int j, int d,
                                          uint32_t raw) {
    const unsigned m = __ballot_sync(0xffffffffu, hit);
    if (!m) return;
    const int leader = __ffs(m) - 1;
    int base = 0;
    if (wl == leader) base = atomicAdd(p.cand_count, __popc(m));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (hit) {
        const int pos = base + __popc(m & ((1u << wl) - 1));
        if (pos < p.cand_cap) {
            Cand cd;
            cd.item = item;
            cd.j = j;
            cd.d = d;
            cd.raw = raw;
            p.cands[pos] = cd;
        }
    }
}

// Null3 correction of a hit of length len with residue counts n[4]
// (score_correction_null3, src/cp9.rs:6516-6528), computed as the host does
// but with the device's log and, for the final FLogsum(0, x), the exact
// log2(1 + 2^-x) instead of the 0.001-step table: used only to decide which
// cells the host must look at, within a margin that covers both differences.
__device__ float null3_approx(const ScanParams &p, const uint32_t *n, int len) {
    float comp[4], sum = 0.0f;
#pragma unroll
    for (int a = 0; a < 4; a++) {
        comp[a] = (float)n[a];
        sum = __fadd_rn(sum, comp[a]);
    }
#pragma unroll
    for (int a = 0; a < 4; a++) comp[a] = sum > 0.0f ? __fdiv_rn(comp[a], sum) : 0.25f;
    float score = 0.0f;
#pragma unroll
    for (int a = 0; a < 4; a++) {
        const double q = (double)__fdiv_rn(comp[a], p.pf_null[a]);
        const double t = (q > 0.0 ? log(q) * 1.44269504 : -1.0e36) * (double)comp[a] * (double)len;
        score = (float)((double)score + t);
    }
    const double om = (double)p.pf_omega;
    score = (float)((double)score + (om > 0.0 ? log(om) * 1.44269504 : -1.0e36));
    const float mx = fmaxf(0.0f, score), mn = fminf(0.0f, score);
    if (mx - mn >= 23.0f) return mx;
    return mx + (float)log2(1.0 + exp2(-(double)(mx - mn)));
}

// Margin of an approximate corrected score: FLogsum's table step (<= 5e-4
// bits) plus the double-precision log differences (relative ~1e-15) plus
// f32 rounding of the sums (a few ulps of |x|), with room to spare.
__device__ __forceinline__ float pf_margin(float x) { return 2.0e-3f + 1.0e-5f * fabsf(x); }

// Report pre-filter of one lane's column (one warp): the greedy report
// (src/cm_nohmm.rs:769-812) walks d ascending and reports a cell when its
// corrected score c(d) is >= cutoff and above every reported score so far,
// i.e. above R(d) = max{c(d') : d' < d, c(d') >= cutoff}, since the largest
// such c(d') is always reported.  With approximate scores c~ within margin
// m of c, a cell with c~(d) + m(d) <= R~(d) - m(R~), or c~(d) + m(d) < cutoff,
// can neither be reported nor change R, where R~ is the maximum of c~(d')
// over the cells with c~(d') - m(d') >= cutoff.  Every other cell with a
// possible score is emitted, and the host replays the exact rule on them.
// Residue counts of j-d+1..j come from a warp prefix sum over d.
template <class S>
__device__ void prefilter_row(const K &k, int l, int step, int wl) {
    const ScanParams &p = *k.p;
    const unsigned FULL = 0xffffffffu;
    const int32_t *ls = k.s.lane + l * LS_W;
    const int j = ls[LS_JB] + step;
    if (ls[LS_ITEM] < 0 || j > ls[LS_JEND] || j < ls[LS_JREPORT]) return;
    const int jrow = min(j - ls[LS_JSTART] + 1, p.W);
    const int dn0 = p.root_dn, dx0 = min(jrow, p.root_dxcap);
    const uint8_t *ring = k.s.ring + l * p.lay.ring_len;
    const uint32_t *row = k.s.prow + l * k.s.bstride;
    const int item = p.item_base + ls[LS_ITEM];
    uint32_t c01 = 0, c23 = 0;  // counts of residues 0,1 / 2,3 in j-d+1..j, 16 bits each
    float run = -INFINITY;
    for (int base = 1; base <= dx0; base += 32) {
        const int d = base + wl;
        const bool in = d <= dx0;
        const int r = in ? ring[(j - d + 1) & k.rmask] : 4;
        uint32_t x01 = (r == 0 ? 1u : 0u) | (r == 1 ? 0x10000u : 0u);
        uint32_t x23 = (r == 2 ? 1u : 0u) | (r == 3 ? 0x10000u : 0u);
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y01 = __shfl_up_sync(FULL, x01, o), y23 = __shfl_up_sync(FULL, x23, o);
            if (wl >= o) {
                x01 += y01;
                x23 += y23;
            }
        }
        x01 += c01;
        x23 += c23;
        c01 = __shfl_sync(FULL, x01, 31);
        c23 = __shfl_sync(FULL, x23, 31);
        uint32_t raw = 0;
        float c = -INFINITY;
        if (in && d >= dn0) {
            raw = row[d];
            const float bits = S::bits(S::ld(row + d));
            if (bits > IMPOSSIBLE_D + 1.0f) {
                c = bits;
                if (p.do_null3) {
                    const uint32_t n[4] = {x01 & 0xffffu, x01 >> 16, x23 & 0xffffu, x23 >> 16};
                    c = __fsub_rn(c, null3_approx(p, n, d));
                }
            }
        }
        const float m = pf_margin(c);
        float inc = (c > -INFINITY && c - m >= p.cutoff) ? c : -INFINITY;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const float y = __shfl_up_sync(FULL, inc, o);
            if (wl >= o) inc = fmaxf(inc, y);
        }
        float ex = __shfl_up_sync(FULL, inc, 1);
        if (wl == 0) ex = -INFINITY;
        ex = fmaxf(ex, run);
        run = fmaxf(run, __shfl_sync(FULL, inc, 31));
        const bool hit = c > -INFINITY && c + m >= p.cutoff && (ex == -INFINITY || c + m > ex - pf_margin(ex));
        emit_cand(p, wl, hit, item, j, d, raw);
    }
}

// TG: the per-state tables stay in global memory (large models); otherwise
// they are copied to shared memory, and the compiler sees shared addresses.
template <bool INS, bool DECK_SMEM, bool TG>
__global__ void __launch_bounds__(512, 1) qdb_scan_kernel(ScanParams p) {
    typedef Sem<INS> S;
    typedef typename S::T T;
    extern __shared__ __align__(16) uint32_t smem[];
    __shared__ int s_fresh[MAX_LANES];
    __shared__ int s_any;
    const SmemLayout &ly = p.lay;
    K k;
    k.p = &p;
    k.nz = p.ilog_nz;
    k.esc_g = p.esc;
    k.fuse_begin = p.fuse_begin;
    k.begin_key = p.begin_key;
    k.root_dn = p.root_dn;
    k.root_dxcap = p.root_dxcap;
    k.W1 = p.W + 1;
    k.s.el = smem + ly.el;
    k.s.tbl = reinterpret_cast<const uint16_t *>(smem + ly.tbl);
    if (TG) {
        // large models: the per-state tables are read from global memory
        // (read-only, cached in L1) instead of being copied to shared memory
        k.s.info = reinterpret_cast<const int4 *>(p.states);
        k.s.wb = p.wb;
        k.s.cb = p.cb;
        k.s.tsc = p.tsc;
        k.s.endsc = p.endsc;
        k.s.escc = p.esc_c;
        k.s.chunks = reinterpret_cast<const int2 *>(p.chunks);
        k.s.lvl = p.level_start;
        k.s.begin = reinterpret_cast<const int4 *>(p.begins);
        k.s.beginsc = p.beginsc;
    } else {
        k.s.info = reinterpret_cast<const int4 *>(smem + ly.info);
        k.s.wb = reinterpret_cast<const int32_t *>(smem + ly.wb);
        k.s.cb = reinterpret_cast<const int32_t *>(smem + ly.cb);
        k.s.tsc = smem + ly.tsc;
        k.s.endsc = smem + ly.endsc;
        k.s.escc = smem + ly.escc;
        k.s.chunks = reinterpret_cast<const int2 *>(smem + ly.chunks);
        k.s.lvl = reinterpret_cast<const int32_t *>(smem + ly.lvl);
        k.s.begin = reinterpret_cast<const int4 *>(smem + ly.begin);
        k.s.beginsc = smem + ly.beginsc;
    }
    k.s.ring = reinterpret_cast<uint8_t *>(smem + ly.ring);
    k.s.lane = reinterpret_cast<int32_t *>(smem + ly.lane);
    k.s.bsv = smem + ly.bsv;
    k.s.bmax = reinterpret_cast<int32_t *>(smem + ly.bmax);
    k.s.prow = smem + ly.prow;
    k.s.bstride = p.root_dxcap + 1;
    k.rmask = ly.ring_len - 1;

    const int tid = threadIdx.x, wl = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;
    const int bs = blockDim.x;
    const int lanes = p.lanes;
    const int W1 = p.W + 1;
    const T ZERO = S::zero();

    // ---- model metadata into shared memory ----
    {
        auto copy32 = [&](int dst, const void *src, int n) {
            const uint32_t *g = reinterpret_cast<const uint32_t *>(src);
            for (int x = tid; x < n; x += bs) smem[dst + x] = __ldg(g + x);
        };
        copy32(ly.el, p.el_sca, p.W + 1);
        if (INS) copy32(ly.tbl, p.ilog, (p.ilog_nz + 2) / 2);  // entries 0..nz, tbl[nz] = 0
        if (!TG) {
            copy32(ly.info, p.states, p.M * 4);
            copy32(ly.wb, p.wb, p.M * 2);
            copy32(ly.cb, p.cb, p.M * 12);
            copy32(ly.tsc, p.tsc, p.M * 6);
            copy32(ly.endsc, p.endsc, p.M);
            copy32(ly.escc, p.esc_c, p.n_esc_c);
            copy32(ly.chunks, p.chunks, p.nchunks * 2);
            copy32(ly.lvl, p.level_start, p.nlev + 1);
            copy32(ly.begin, p.begins, p.nbegin * 4);
            copy32(ly.beginsc, p.beginsc, p.nbegin);
        }
        if (INS && p.fuse_begin) {
            copy32(ly.bsv, p.beginsc_all, p.M);
            for (int x = tid; x < lanes * (p.root_dxcap + 1); x += bs)
                k.s.bmax[x] = p.begin_key ? INT32_MIN : -INFTY_D;
        }
        if (tid < MAX_LANES * LS_W) k.s.lane[tid] = tid % LS_W == LS_ITEM ? -1 : 0;
    }
    uint32_t *deck_base = DECK_SMEM ? smem + ly.deck
                                    : p.deck_global + (size_t)blockIdx.x * (size_t)lanes * (size_t)p.deck_stride;
    const int64_t deck_stride = DECK_SMEM ? p.deck_elems : p.deck_stride;
    const int rw = max(0, p.root_dxcap - p.root_dn + 1);
    // per-warp walk over units (ci, l): start (u_c0, u_l0), stride (u_dc, u_dl)
    const int u_l0 = warp % lanes, u_c0 = warp / lanes;
    const int u_dl = nwarps % lanes, u_dc = nwarps / lanes;
    // per-thread walk over root cells (l, d): start (r_l0, r_d0), stride (r_dl, r_dd)
    const int r_l0 = rw > 0 ? tid / rw : 0, r_d0 = rw > 0 ? tid % rw : 0;
    const int r_dl = rw > 0 ? bs / rw : 0, r_dd = rw > 0 ? bs % rw : 0;

    for (;;) {
        __syncthreads();
        // ---- refill lanes whose item ended ----
        if (tid == 0) {
            int any = 0;
            for (int l = 0; l < lanes; l++) {
                int32_t *ls = k.s.lane + l * LS_W;
                s_fresh[l] = 0;
                if (ls[LS_ITEM] == -1 || (ls[LS_ITEM] >= 0 && ls[LS_JB] > ls[LS_JEND])) {
                    int it = atomicAdd(p.next_item, 1);
                    if (it < p.nitems) {
                        WorkItem wi = p.items[it];
                        ls[LS_ITEM] = it;
                        ls[LS_JB] = wi.jstart;
                        ls[LS_JSTART] = wi.jstart;
                        ls[LS_JEND] = wi.jend;
                        ls[LS_JREPORT] = wi.jreport;
                        ls[LS_OFFLO] = (int32_t)(uint32_t)((uint64_t)wi.dsq_off & 0xffffffffu);
                        ls[LS_OFFHI] = (int32_t)(uint32_t)((uint64_t)wi.dsq_off >> 32);
                        ls[LS_JM] = wi.jstart % W1;
                        s_fresh[l] = 1;
                    } else {
                        ls[LS_ITEM] = -2;
                    }
                }
                if (ls[LS_ITEM] >= 0) any = 1;
            }
            s_any = any;
        }
        __syncthreads();
        if (!s_any) break;
        // ---- fresh decks: fill, then the d = 0 base cells ----
        bool any_fresh = false;
        for (int l = 0; l < lanes; l++) {
            if (!s_fresh[l]) continue;
            any_fresh = true;
            uint32_t *dk = deck_base + (size_t)l * deck_stride;
            for (int64_t x = tid; x < p.deck_elems; x += bs) S::st(dk + x, ZERO);
        }
        if (any_fresh) {
            __syncthreads();
            for (int l = 0; l < lanes; l++) {
                if (!s_fresh[l]) continue;
                uint32_t *dk = deck_base + (size_t)l * deck_stride;
                for (int x = tid; x < p.ninit; x += bs) dk[__ldg(p.init_off + x)] = __ldg(p.init_val + x);
            }
        }
        // ---- residues of this block into the lane rings ----
        for (int t = tid; t < lanes * COL_BLOCK; t += bs) {
            int l = t / COL_BLOCK, q = t % COL_BLOCK;
            const int32_t *ls = k.s.lane + l * LS_W;
            int x = ls[LS_JB] + q;
            if (ls[LS_ITEM] >= 0 && x <= ls[LS_JEND]) {
                uint64_t off = (uint64_t)(uint32_t)ls[LS_OFFLO] | ((uint64_t)(uint32_t)ls[LS_OFFHI] << 32);
                int c = __ldg(p.dsq + off + x);
                k.s.ring[l * ly.ring_len + (x & k.rmask)] = (uint8_t)(c > 17 ? 17 : c);
            }
        }
        __syncthreads();

        for (int step = 0; step < COL_BLOCK; step++) {
            // ---- levels ----
            for (int lev = 0; lev < p.nlev; lev++) {
                const int c0 = k.s.lvl[lev], nch = k.s.lvl[lev + 1] - c0;
                // unit u = ci * lanes + l, walked without divisions
                int l = u_l0, ci = u_c0;
                for (; ci < nch; l += u_dl, ci += u_dc) {
                    if (l >= lanes) {
                        l -= lanes;
                        ci++;
                        if (ci >= nch) break;
                    }
                    const int32_t *ls = k.s.lane + l * LS_W;
                    const int j = ls[LS_JB] + step;
                    if (ls[LS_ITEM] < 0 || j > ls[LS_JEND]) continue;
                    Lane L;
                    L.l = l;
                    L.deck = deck_base + (size_t)l * deck_stride;
                    L.ring = k.s.ring + l * ly.ring_len;
                    L.j = j;
                    L.par = j & 1;
                    int jm = ls[LS_JM] + step;
                    while (jm >= W1) jm -= W1;
                    L.jm = jm;
                    L.jrow = min(j - ls[LS_JSTART] + 1, p.W);
                    const int2 ch = k.s.chunks[c0 + ci];
                    const SInfo sv = unpack(k.s.info[ch.x]);
                    if (ch.y < 0)
                        do_il<S>(k, L, ch.x, sv, wl);
                    else if (sv.type == 8)
                        do_bif_chunk<S>(k, L, ch.x, sv, ch.y, wl);
                    else
                        do_chunk<S>(k, L, ch.x, sv, ch.y, wl);
                }
                __syncthreads();
            }
            // ---- ROOT_S, local begins, candidates ----
            int rl = r_l0, rd0 = r_d0;
            for (int tb = 0; tb < lanes * rw; tb += bs, rl += r_dl, rd0 += r_dd) {
                if (rd0 >= rw) {
                    rd0 -= rw;
                    rl++;
                }
                bool hit = false;
                T a = ZERO;
                int l = rl, d = p.root_dn + rd0, j = 0;
                if (rl < lanes) {
                    const int32_t *ls = k.s.lane + l * LS_W;
                    j = ls[LS_JB] + step;
                    if (ls[LS_ITEM] >= 0 && j <= ls[LS_JEND]) {
                        const int jrow = min(j - ls[LS_JSTART] + 1, p.W);
                        const int dx0 = min(jrow, p.root_dxcap);
                        if (d <= dx0) {
                            const uint32_t *deck = deck_base + (size_t)l * deck_stride;
                            const int par = j & 1;
                            int jm = ls[LS_JM] + step;
                            while (jm >= W1) jm -= W1;
#pragma unroll
                            for (int yo = 0; yo < 6; yo++) {
                                if (yo < p.root_cnum) {
                                    T term = S::add(S::ld(deck + k.s.cb[2 * yo + par] + d), S::ld(k.s.tsc + yo));
                                    a = yo == 0 ? S::comb(ZERO, term, k.s.tbl, k.nz) : S::comb(a, term, k.s.tbl, k.nz);
                                }
                            }
                            if (INS && p.fuse_begin) {
                                int32_t *bm = k.s.bmax + l * k.s.bstride + d;
                                const T cand = (T)*bm;
                                *bm = p.begin_key ? INT32_MIN : -INFTY_D;
                                if (begin_less<S>(p.begin_key, a, cand)) a = cand;
                            } else if (p.local) {
                                for (int b = 0; b < p.nbegin; b++) {
                                    const int4 bd = k.s.begin[b];
                                    const int dn = (int16_t)(bd.w & 0xffff), dxc = (int16_t)((uint32_t)bd.w >> 16);
                                    if (d < dn || d > dxc) continue;
                                    int rb;
                                    if (bd.y == bd.z) {  // single slot, or a BEGL ring
                                        const SInfo sy = unpack(k.s.info[bd.x]);
                                        rb = (sy.flags & SF_BEGL) ? bd.y + jm * sy.span : bd.y;
                                    } else {
                                        rb = par ? bd.z : bd.y;
                                    }
                                    T cand = S::add(S::ld(deck + rb + d), S::ld(k.s.beginsc + b));
                                    if (begin_less<S>(p.begin_key, a, cand)) a = cand;
                                }
                            }
                            if (p.prefilter) {
                                k.s.prow[l * k.s.bstride + d] = S::u(a);
                            } else if (j >= ls[LS_JREPORT]) {
                                float sc = S::bits(a);
                                hit = sc >= p.cutoff && sc > IMPOSSIBLE_D + 1.0f;
                            }
                        }
                    }
                }
                emit_cand(p, wl, hit, hit ? p.item_base + k.s.lane[l * LS_W + LS_ITEM] : 0, j, d, S::u(a));
            }
            if (p.prefilter) {
                __syncthreads();
                for (int l = warp; l < lanes; l += nwarps) prefilter_row<S>(k, l, step, wl);
            }
            if (INS && p.fuse_begin) __syncthreads();  // ROOT-row resets before the next column's posts
        }
        // advance every live lane by one block
        __syncthreads();
        if (tid < lanes) {
            int32_t *ls = k.s.lane + tid * LS_W;
            if (ls[LS_ITEM] >= 0) {
                ls[LS_JB] += COL_BLOCK;
                ls[LS_JM] = (ls[LS_JM] + COL_BLOCK) % W1;
            }
        }
    }
}

template <bool INS, bool DS, bool TG>
static cudaError_t launch_t(const ScanParams &p, int ctas, int threads, cudaStream_t s) {
    auto kern = qdb_scan_kernel<INS, DS, TG>;
    size_t smem = (size_t)p.lay.words * 4;
    cudaError_t e = cmx::allow_max_dynamic_smem(kern);
    if (e != cudaSuccess) return e;
    kern<<<ctas, threads, smem, s>>>(p);
    return cudaGetLastError();
}

template <bool INS, bool DS, bool TG>
static int occupancy_t(const ScanParams &p, int threads) {
    int n = 0;
    auto kern = qdb_scan_kernel<INS, DS, TG>;
    size_t smem = (size_t)p.lay.words * 4;
    if (cmx::allow_max_dynamic_smem(kern) != cudaSuccess) return 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kern, threads, smem) != cudaSuccess) return 0;
    return n;
}

}  // namespace dev

SmemLayout scan_layout(const ScanParams &p, int lanes, bool deck_smem) {
    SmemLayout L{};
    int64_t w = 0;
    auto take = [&](int64_t n) {
        int64_t o = w;
        w += (n + 3) & ~(int64_t)3;  // keep 16-byte alignment
        return (int)o;
    };
    L.el = take(p.W + 1);
    L.tbl = take(p.inside ? (p.ilog_nz + 2) / 2 : 0);
    const int64_t g = p.tables_global ? 0 : 1;  // per-state tables in shared memory?
    L.info = take(g * p.M * 4);
    L.wb = take(g * p.M * 2);
    L.cb = take(g * p.M * 12);
    L.tsc = take(g * p.M * 6);
    L.endsc = take(g * p.M);
    L.escc = take(g * p.n_esc_c);
    L.chunks = take(g * p.nchunks * 2);
    L.lvl = take(g * (p.nlev + 1));
    L.begin = take(g * p.nbegin * 4);
    L.beginsc = take(g * p.nbegin);
    int r = 1;
    while (r < p.W + 64) r <<= 1;
    L.ring_len = r;
    L.ring = take((int64_t)lanes * r / 4);
    L.lane = take((int64_t)MAX_LANES * 8);
    L.bsv = take(p.fuse_begin ? p.M : 0);
    L.bmax = take(p.fuse_begin ? (int64_t)lanes * (p.root_dxcap + 1) : 0);
    L.prow = take(p.prefilter ? (int64_t)lanes * (p.root_dxcap + 1) : 0);
    L.deck = take(deck_smem ? (int64_t)lanes * p.deck_elems : 0);
    L.words = w;
    return L;
}

int scan_occupancy(const ScanParams &p, int threads) {
    const int sel = (p.inside ? 4 : 0) | (p.deck_smem ? 2 : 0) | (p.tables_global ? 1 : 0);
    switch (sel) {
    case 0: return dev::occupancy_t<false, false, false>(p, threads);
    case 1: return dev::occupancy_t<false, false, true>(p, threads);
    case 2: return dev::occupancy_t<false, true, false>(p, threads);
    case 3: return dev::occupancy_t<false, true, true>(p, threads);
    case 4: return dev::occupancy_t<true, false, false>(p, threads);
    case 5: return dev::occupancy_t<true, false, true>(p, threads);
    case 6: return dev::occupancy_t<true, true, false>(p, threads);
    default: return dev::occupancy_t<true, true, true>(p, threads);
    }
}

cudaError_t scan_launch(const ScanParams &p, int ctas, int threads, cudaStream_t s) {
    const int sel = (p.inside ? 4 : 0) | (p.deck_smem ? 2 : 0) | (p.tables_global ? 1 : 0);
    switch (sel) {
    case 0: return dev::launch_t<false, false, false>(p, ctas, threads, s);
    case 1: return dev::launch_t<false, false, true>(p, ctas, threads, s);
    case 2: return dev::launch_t<false, true, false>(p, ctas, threads, s);
    case 3: return dev::launch_t<false, true, true>(p, ctas, threads, s);
    case 4: return dev::launch_t<true, false, false>(p, ctas, threads, s);
    case 5: return dev::launch_t<true, false, true>(p, ctas, threads, s);
    case 6: return dev::launch_t<true, true, false>(p, ctas, threads, s);
    default: return dev::launch_t<true, true, true>(p, ctas, threads, s);
    }
}

}  // namespace cmx
