// QDB-banded CYK / Inside window scanner for sm_100a.
//
// One persistent CTA scans one work item at a time: a piece of a window plus
// W-1 warm-up columns, pulled from a cost-ordered device queue.  A cell (j,d)
// depends only on residues j-d+1..j, so a piece started W-1 columns early
// reproduces the reference's cells bit for bit (src/cm_nohmm.rs:549-763
// computes them with jrow = min(j-i0+1, W)).
//
// Per column j the CTA walks the plan's levels:
//   level 0   every right emitter (MP, MR, IR).  They read only column j-1
//             (jp_y = prv, src/cm_nohmm.rs:575), so all of them are
//             independent and run in one phase;
//   level l   states whose same-column children sit in levels < l;
//   root      ROOT_S transitions, local begins (MAX in both semirings,
//             src/cm_nohmm.rs:700-746) and candidate emission.
// Warps take (state, 32 cells) chunks; lanes are consecutive d.  Cells are
// evaluated with the reference's operand order (reduce_c_order,
// src/cm_nohmm.rs:187-242, for emitters, S and D states; natural child order
// for BEGL_S, :601-611; ascending k for bifurcations) so integer ILogsum
// results are bit-identical; f32 adds use __fadd_rn (no contraction).
//
// IL states read their own cell d-1 (self loop, src/cm_nohmm.rs:622-649), a
// serial chain in d.  A warp resolves it by blocked fixed-point iteration:
// lane l owns a block of consecutive d, walks it serially from an incoming
// value, and passes its last value to lane l+1; the warp repeats until no
// incoming value changes.  The step x -> comb(c, x + t0) + e is monotone, so
// the fixed point is the serial result exactly, and 33 rounds always reach it.
//
// Decks: right emitters keep two column slots (j & 1), BEGL_S states a ring
// of W+1 columns, every other state one slot that level 0 of column j reads
// (as column j-1) before levels >= 1 overwrite it.  All decks live in shared
// memory when they fit; otherwise in a per-CTA region of global memory.
#include <cuda_runtime.h>
#include <cstdint>

#include "qdb_kernel.h"

namespace cmx {
namespace dev {

constexpr int INFTY_D = 987654321;
constexpr float IMPOSSIBLE_D = -1.0e36f;

template <bool INS>
struct Sem;

template <>
struct Sem<false> {  // CYK: f32, ESL_MAX
    typedef float T;
    __device__ static __forceinline__ T zero() { return IMPOSSIBLE_D; }
    __device__ static __forceinline__ T add(T a, T b) { return __fadd_rn(a, b); }
    __device__ static __forceinline__ T comb(T a, T b, const uint16_t *, int) { return a >= b ? a : b; }
    __device__ static __forceinline__ T ld(const uint32_t *p) { return __uint_as_float(*p); }
    __device__ static __forceinline__ T ldg(const uint32_t *p) { return __uint_as_float(__ldg(p)); }
    __device__ static __forceinline__ void st(uint32_t *p, T x) { *p = __float_as_uint(x); }
    __device__ static __forceinline__ uint32_t u(T x) { return __float_as_uint(x); }
    __device__ static __forceinline__ float bits(T x) { return x; }
};

template <>
struct Sem<true> {  // Inside: i32 wrapping adds, ILogsum
    typedef int32_t T;
    __device__ static __forceinline__ T zero() { return -INFTY_D; }
    __device__ static __forceinline__ T add(T a, T b) { return (int32_t)((uint32_t)a + (uint32_t)b); }
    // ILogsum (src/cp9.rs:65-75): max + tbl[max-min]; the table is stored up
    // to its last nonzero entry (nz), beyond which it adds 0 like the rule
    // (max-min) >= LOGSUM_TBL does.
    __device__ static __forceinline__ T comb(T a, T b, const uint16_t *tbl, int nz) {
        int32_t mx = a > b ? a : b;
        if (mx < -INFTY_D) mx = -INFTY_D;
        int32_t mn = a < b ? a : b;
        uint32_t diff = (uint32_t)mx - (uint32_t)mn;
        if (mn <= -INFTY_D || diff >= (uint32_t)nz) return mx;
        return (int32_t)((uint32_t)mx + (uint32_t)tbl[diff]);
    }
    __device__ static __forceinline__ T ld(const uint32_t *p) { return (int32_t)*p; }
    __device__ static __forceinline__ T ldg(const uint32_t *p) { return (int32_t)__ldg(p); }
    __device__ static __forceinline__ void st(uint32_t *p, T x) { *p = (uint32_t)x; }
    __device__ static __forceinline__ uint32_t u(T x) { return (uint32_t)x; }
    __device__ static __forceinline__ float bits(T x) {
        return x == -INFTY_D ? IMPOSSIBLE_D : (float)((double)x / 1000.0);
    }
};

struct SInfo {  // the first 16 bytes of StateDev
    int32_t base;
    int16_t dn, dxcap, width;
    uint8_t flags, type;
    int16_t cfirst, cnum;
};

__device__ __forceinline__ SInfo load_info(const StateDev *st, int v) {
    int4 q = __ldg(reinterpret_cast<const int4 *>(st + v));
    SInfo s;
    s.base = q.x;
    s.dn = (int16_t)(q.y & 0xffff);
    s.dxcap = (int16_t)((uint32_t)q.y >> 16);
    s.width = (int16_t)(q.z & 0xffff);
    s.flags = (uint8_t)(((uint32_t)q.z >> 16) & 0xff);
    s.type = (uint8_t)((uint32_t)q.z >> 24);
    s.cfirst = (int16_t)(q.w & 0xffff);
    s.cnum = (int16_t)((uint32_t)q.w >> 16);
    return s;
}

// Residue code at frame position x.  Codes above 17 (not produced by the
// digitiser) read as 17 (missing), so a malformed buffer cannot index past an
// emission row; the host rejects such buffers before launch when it can.
__device__ __forceinline__ int res(const uint8_t *frame, int x) {
    int c = __ldg(frame + x);
    return c > 17 ? 17 : c;
}

__device__ __forceinline__ int state_delta(int t) {
    return t == 1 ? 2 : (t >= 2 && t <= 5) ? 1 : 0;  // MP 2; ML MR IL IR 1
}
__device__ __forceinline__ bool right_em(int t) { return t == 1 || t == 3 || t == 5; }

// Value of cell idx of state Y in column slot `slot` (parity for two-slot
// states, ring column for BEGL_S, ignored otherwise).
template <class S>
__device__ __forceinline__ typename S::T rd(const SInfo &Y, const uint32_t *deck, int slot, int idx,
                                            const uint32_t *init0, int y) {
    if ((unsigned)(idx - Y.dn) <= (unsigned)(Y.dxcap - Y.dn) && Y.width > 0) {
        int so = (Y.flags & (SF_TWO_SLOT | SF_BEGL)) ? slot * Y.width : 0;
        return S::ld(deck + Y.base + so + idx);
    }
    if (idx == 0) return S::ldg(init0 + y);
    return S::zero();
}

// reduce_c_order (src/cm_nohmm.rs:187-242); t[] are the child terms.
template <class S>
__device__ __forceinline__ typename S::T reduce_c(int cnum, const typename S::T *t, typename S::T init,
                                                  const uint16_t *tb, int nz) {
    typedef typename S::T T;
    T s;
    switch (cnum) {
    case 1: s = S::comb(init, t[0], tb, nz); break;
    case 2: s = S::comb(S::comb(t[1], init, tb, nz), t[0], tb, nz); break;
    case 3: s = S::comb(S::comb(S::comb(t[2], t[1], tb, nz), init, tb, nz), t[0], tb, nz); break;
    case 4:
        s = S::comb(t[3], t[2], tb, nz);
        s = S::comb(s, init, tb, nz);
        s = S::comb(s, t[1], tb, nz);
        s = S::comb(s, t[0], tb, nz);
        break;
    case 5:
        s = S::comb(t[4], t[3], tb, nz);
        s = S::comb(s, init, tb, nz);
        s = S::comb(s, t[1], tb, nz);
        s = S::comb(s, t[2], tb, nz);
        s = S::comb(s, t[0], tb, nz);
        break;
    case 6:
        s = S::comb(t[5], init, tb, nz);
        s = S::comb(s, t[4], tb, nz);
        s = S::comb(s, t[3], tb, nz);
        s = S::comb(s, t[2], tb, nz);
        s = S::comb(s, t[1], tb, nz);
        s = S::comb(s, t[0], tb, nz);
        break;
    default:
        s = init;
        for (int q = 0; q < cnum; q++) s = S::comb(s, t[q], tb, nz);
    }
    return s;
}

// The same order with the self term t[0] left out: the IL step is then
// comb(c, x + t0) (t[0] is combined last for every cnum).
template <class S>
__device__ __forceinline__ typename S::T reduce_c_noself(int cnum, const typename S::T *t, typename S::T init,
                                                         const uint16_t *tb, int nz) {
    typedef typename S::T T;
    T s;
    switch (cnum) {
    case 1: s = init; break;
    case 2: s = S::comb(t[1], init, tb, nz); break;
    case 3: s = S::comb(S::comb(t[2], t[1], tb, nz), init, tb, nz); break;
    case 4:
        s = S::comb(t[3], t[2], tb, nz);
        s = S::comb(s, init, tb, nz);
        s = S::comb(s, t[1], tb, nz);
        break;
    case 5:
        s = S::comb(t[4], t[3], tb, nz);
        s = S::comb(s, init, tb, nz);
        s = S::comb(s, t[1], tb, nz);
        s = S::comb(s, t[2], tb, nz);
        break;
    case 6:
        s = S::comb(t[5], init, tb, nz);
        s = S::comb(s, t[4], tb, nz);
        s = S::comb(s, t[3], tb, nz);
        s = S::comb(s, t[2], tb, nz);
        s = S::comb(s, t[1], tb, nz);
        break;
    default:
        s = init;
        for (int q = 1; q < cnum; q++) s = S::comb(s, t[q], tb, nz);
    }
    return s;
}

struct Ctx {
    const ScanParams *p;
    uint32_t *deck;
    const uint32_t *el_sca;   // shared
    const uint16_t *tbl;      // shared ILogsum table (Inside)
    const uint8_t *frame;     // window frame of the current item
    int j, cur, prv, jm, jrow;
};

// Children terms of cell (v, d) for a non-B state: terms[yo] = child + tsc.
template <class S>
__device__ __forceinline__ void child_terms(const Ctx &c, const SInfo &sv, int v, int idx, int slot,
                                            typename S::T *terms, int first) {
    const ScanParams &p = *c.p;
    for (int yo = first; yo < sv.cnum; yo++) {
        int y = sv.cfirst + yo;
        SInfo sy = load_info(p.states, y);
        terms[yo] = S::add(rd<S>(sy, c.deck, slot, idx, p.init0, y), S::ldg(p.tsc + v * 6 + yo));
    }
}

template <class S>
__device__ __forceinline__ typename S::T init_sc(const Ctx &c, const SInfo &sv, int v, int idx) {
    if (sv.flags & SF_ENDSC) return S::add(S::ld(c.el_sca + idx), S::ldg(c.p->endsc + v));
    return S::zero();
}

// One warp-wide chunk of an ordinary state (not B, not IL).
template <class S>
__device__ __forceinline__ void do_chunk(const Ctx &c, int v, int d0, int lane) {
    typedef typename S::T T;
    const ScanParams &p = *c.p;
    SInfo sv = load_info(p.states, v);
    int d = d0 + lane;
    int dx = min(c.jrow, (int)sv.dxcap);
    if (d > dx) return;
    int t = sv.type;
    int sd = state_delta(t);
    bool rem = right_em(t);
    int slot_y = rem ? c.prv : c.cur;
    int idx = d - sd;
    T terms[6];
    child_terms<S>(c, sv, v, idx, slot_y, terms, 0);
    T sc;
    if (sv.flags & SF_BEGL) {
        // BEGL_S folds its children in natural order (src/cm_nohmm.rs:601-611)
        sc = init_sc<S>(c, sv, v, idx);
        for (int yo = 0; yo < sv.cnum; yo++) sc = S::comb(sc, terms[yo], c.tbl, p.ilog_nz);
    } else {
        sc = reduce_c<S>(sv.cnum, terms, init_sc<S>(c, sv, v, idx), c.tbl, p.ilog_nz);
    }
    int esc_off = v * 324;
    if (t == 2 || t == 4) {  // ML, IL: residue i = j-d+1
        sc = S::add(sc, S::ldg(p.esc + esc_off + res(c.frame, c.j - d + 1)));
    } else if (t == 3 || t == 5) {  // MR, IR: residue j
        sc = S::add(sc, S::ldg(p.esc + esc_off + res(c.frame, c.j)));
    } else if (t == 1) {  // MP
        sc = S::add(sc, S::ldg(p.esc + esc_off + res(c.frame, c.j - d + 1) * 18 + res(c.frame, c.j)));
    }
    int so;
    if (sv.flags & SF_BEGL)
        so = c.jm * sv.width;
    else if (sv.flags & SF_TWO_SLOT)
        so = c.cur * sv.width;
    else
        so = 0;
    S::st(c.deck + sv.base + so + d, sc);
}

// Bifurcation chunk: alpha[v][d] = init (+) over k ascending of
// BEGL(j-k, d-k) + BEGR(j, k) (src/cm_nohmm.rs:578-600).
template <class S>
__device__ __forceinline__ void do_bif_chunk(const Ctx &c, int v, int d0, int lane) {
    typedef typename S::T T;
    const ScanParams &p = *c.p;
    SInfo sv = load_info(p.states, v);
    int d = d0 + lane;
    int dx = min(c.jrow, (int)sv.dxcap);
    if (d > dx) return;
    int4 q2 = __ldg(reinterpret_cast<const int4 *>(p.states + v) + 1);
    int kdn_y = (int16_t)(q2.x & 0xffff), kdx_y = (int16_t)((uint32_t)q2.x >> 16);
    int kdn_w = (int16_t)(q2.y & 0xffff), kdx_w = (int16_t)((uint32_t)q2.y >> 16);
    int wl = sv.cfirst, y = sv.cnum;
    SInfo sw = load_info(p.states, wl);
    SInfo sy = load_info(p.states, y);
    int kmin = max(0, max(kdn_y, d - kdx_w));
    int kmax = min(kdx_y, d - kdn_w);
    T sc = init_sc<S>(c, sv, v, d);
    const int W1 = p.W + 1;
    int col = c.jm - kmin;
    if (col < 0) col += W1;
    for (int kk = kmin; kk <= kmax; kk++) {
        T left = rd<S>(sw, c.deck, col, d - kk, p.init0, wl);
        T right = rd<S>(sy, c.deck, c.cur, kk, p.init0, y);
        sc = S::comb(sc, S::add(left, right), c.tbl, p.ilog_nz);
        col = col == 0 ? W1 - 1 : col - 1;
    }
    int so = (sv.flags & SF_TWO_SLOT) ? c.cur * sv.width : 0;
    S::st(c.deck + sv.base + so + d, sc);
}

// IL state: whole band by one warp (see the file comment).
template <class S>
__device__ __forceinline__ void do_il(const Ctx &c, int v, int lane) {
    typedef typename S::T T;
    const ScanParams &p = *c.p;
    SInfo sv = load_info(p.states, v);
    const int dn = sv.dn;
    const int dx = min(c.jrow, (int)sv.dxcap);
    const int n = dx - dn + 1;
    if (n <= 0) return;
    const T t0 = S::ldg(p.tsc + v * 6);
    const int esc_off = v * 324;
    uint32_t *dst = c.deck + sv.base;  // IL is single-slot
    const int k = (n + 31) >> 5;
    if (k <= IL_KMAX) {
        T cv[IL_KMAX], ev[IL_KMAX], xv[IL_KMAX];
        const int dbeg = dn + lane * k;
#pragma unroll
        for (int q = 0; q < IL_KMAX; q++) {
            int d = dbeg + q;
            cv[q] = S::zero();
            ev[q] = S::zero();
            xv[q] = S::zero();
            if (q < k && d <= dx) {
                int idx = d - 1;
                T terms[6];
                child_terms<S>(c, sv, v, idx, c.cur, terms, 1);
                cv[q] = reduce_c_noself<S>(sv.cnum, terms, init_sc<S>(c, sv, v, idx), c.tbl, p.ilog_nz);
                ev[q] = S::ldg(p.esc + esc_off + res(c.frame, c.j - d + 1));
            }
        }
        // x at d = dn-1 is an unwritten cell of the emitter: zero.
        T xin = S::zero(), xin_prev = S::zero(), xlast = S::zero();
        for (int it = 0; it < 34; it++) {
            T x = xin;
#pragma unroll
            for (int q = 0; q < IL_KMAX; q++) {
                if (q < k && dbeg + q <= dx) {
                    x = S::add(S::comb(cv[q], S::add(x, t0), c.tbl, p.ilog_nz), ev[q]);
                    xv[q] = x;
                }
            }
            xlast = x;
            bool same = S::u(xin) == S::u(xin_prev);
            if (it > 0 && __all_sync(0xffffffffu, same)) break;
            xin_prev = xin;
            T up = __shfl_up_sync(0xffffffffu, xlast, 1);
            xin = lane == 0 ? S::zero() : up;
        }
#pragma unroll
        for (int q = 0; q < IL_KMAX; q++) {
            int d = dbeg + q;
            if (q < k && d <= dx) S::st(dst + d, xv[q]);
        }
    } else {
        // wide band: compute c in parallel into the deck, then one lane walks d
        for (int d = dn + lane; d <= dx; d += 32) {
            int idx = d - 1;
            T terms[6];
            child_terms<S>(c, sv, v, idx, c.cur, terms, 1);
            S::st(dst + d, reduce_c_noself<S>(sv.cnum, terms, init_sc<S>(c, sv, v, idx), c.tbl, p.ilog_nz));
        }
        __syncwarp();
        if (lane == 0) {
            T x = S::zero();
            for (int d = dn; d <= dx; d++) {
                T e = S::ldg(p.esc + esc_off + res(c.frame, c.j - d + 1));
                x = S::add(S::comb(S::ld(dst + d), S::add(x, t0), c.tbl, p.ilog_nz), e);
                S::st(dst + d, x);
            }
        }
        __syncwarp();
    }
}

template <bool INS, bool DECK_SMEM>
__global__ void __launch_bounds__(512) qdb_scan_kernel(ScanParams p) {
    typedef Sem<INS> S;
    typedef typename S::T T;
    extern __shared__ __align__(16) uint32_t smem[];
    uint32_t *s_el = smem;                                     // W+1
    uint16_t *s_tbl = reinterpret_cast<uint16_t *>(smem + (p.W + 1));
    const int tbl_words = INS ? (p.ilog_nz + 1) / 2 : 0;
    uint32_t *s_deck = smem + (p.W + 1) + tbl_words;
    __shared__ int s_item;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;
    for (int k = tid; k <= p.W; k += blockDim.x) s_el[k] = __ldg(p.el_sca + k);
    if (INS)
        for (int k = tid; k < p.ilog_nz; k += blockDim.x) s_tbl[k] = __ldg(p.ilog + k);

    Ctx c;
    c.p = &p;
    c.deck = DECK_SMEM ? s_deck : p.deck_global + (size_t)blockIdx.x * (size_t)p.deck_stride;
    c.el_sca = s_el;
    c.tbl = s_tbl;
    const T ZERO = S::zero();
    const int W1 = p.W + 1;

    for (;;) {
        __syncthreads();
        if (tid == 0) s_item = atomicAdd(p.next_item, 1);
        __syncthreads();
        const int it = s_item;
        if (it >= p.nitems) break;
        const WorkItem wi = p.items[it];
        for (int64_t k = tid; k < p.deck_elems; k += blockDim.x) S::st(c.deck + k, ZERO);
        __syncthreads();
        c.frame = p.dsq + wi.dsq_off;
        int jm = wi.jstart % W1;
        for (int j = wi.jstart; j <= wi.jend; j++) {
            c.j = j;
            c.cur = j & 1;
            c.prv = c.cur ^ 1;
            c.jm = jm;
            c.jrow = min(j - wi.jstart + 1, p.W);
            for (int l = 0; l < p.nlev; l++) {
                const int c0 = __ldg(p.level_start + l), c1 = __ldg(p.level_start + l + 1);
                for (int ci = c0 + warp; ci < c1; ci += nwarps) {
                    ChunkDev ch = p.chunks[ci];
                    int t = p.states[ch.v].type;
                    if (ch.d0 < 0)
                        do_il<S>(c, ch.v, lane);
                    else if (t == 8)
                        do_bif_chunk<S>(c, ch.v, ch.d0, lane);
                    else
                        do_chunk<S>(c, ch.v, ch.d0, lane);
                }
                __syncthreads();
            }
            // ROOT_S, local begins, candidates
            const int dx0 = min(c.jrow, p.root_dxcap);
            const bool report = j >= wi.jreport;
            for (int dbase = p.root_dn; dbase <= dx0; dbase += blockDim.x) {
                const int d = dbase + tid;
                bool hit = false;
                T a = ZERO;
                if (d <= dx0) {
                    for (int yo = 0; yo < p.root_cnum; yo++) {
                        int y = p.root_cfirst + yo;
                        SInfo sy = load_info(p.states, y);
                        T term = S::add(rd<S>(sy, c.deck, c.cur, d, p.init0, y), S::ldg(p.tsc + yo));
                        a = yo == 0 ? S::comb(ZERO, term, c.tbl, p.ilog_nz) : S::comb(a, term, c.tbl, p.ilog_nz);
                    }
                    if (p.local) {
                        for (int b = 0; b < p.nbegin; b++) {
                            int y = __ldg(p.begin_states + b);
                            SInfo sy = load_info(p.states, y);
                            int hi = min(dx0, (int)sy.dxcap);
                            if (d < sy.dn || d > hi) continue;
                            T val = rd<S>(sy, c.deck, (sy.flags & SF_BEGL) ? jm : c.cur, d, p.init0, y);
                            T cand = S::add(val, S::ldg(p.beginsc + y));
                            if (a < cand) a = cand;
                        }
                    }
                    if (report) {
                        float sc = S::bits(a);
                        hit = sc >= p.cutoff && sc > IMPOSSIBLE_D + 1.0f;
                    }
                }
                unsigned m = __ballot_sync(0xffffffffu, hit);
                if (m) {
                    int leader = __ffs(m) - 1;
                    int base = 0;
                    if (lane == leader) base = atomicAdd(p.cand_count, __popc(m));
                    base = __shfl_sync(0xffffffffu, base, leader);
                    if (hit) {
                        int pos = base + __popc(m & ((1u << lane) - 1));
                        if (pos < p.cand_cap) {
                            Cand cd;
                            cd.item = p.item_base + it;
                            cd.j = j;
                            cd.d = d;
                            cd.raw = S::u(a);
                            p.cands[pos] = cd;
                        }
                    }
                }
            }
            jm = jm + 1 == W1 ? 0 : jm + 1;
        }
    }
}

template <bool INS, bool DS>
static cudaError_t launch_t(const ScanParams &p, int ctas, int threads, size_t smem, cudaStream_t s) {
    auto kern = qdb_scan_kernel<INS, DS>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    kern<<<ctas, threads, smem, s>>>(p);
    return cudaGetLastError();
}

template <bool INS, bool DS>
static int occupancy_t(int threads, size_t smem) {
    int n = 0;
    auto kern = qdb_scan_kernel<INS, DS>;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) return 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kern, threads, smem) != cudaSuccess) return 0;
    return n;
}

}  // namespace dev

size_t scan_smem_bytes(const ScanParams &p, bool deck_smem) {
    size_t b = (size_t)(p.W + 1) * 4;
    if (p.inside) b += (size_t)((p.ilog_nz + 1) / 2) * 4;
    if (deck_smem) b += (size_t)p.deck_elems * 4;
    return b;
}

int scan_occupancy(const ScanParams &p, bool deck_smem, int threads) {
    size_t smem = scan_smem_bytes(p, deck_smem);
    if (p.inside)
        return deck_smem ? dev::occupancy_t<true, true>(threads, smem) : dev::occupancy_t<true, false>(threads, smem);
    return deck_smem ? dev::occupancy_t<false, true>(threads, smem) : dev::occupancy_t<false, false>(threads, smem);
}

cudaError_t scan_launch(const ScanParams &p, bool deck_smem, int ctas, int threads, cudaStream_t s) {
    size_t smem = scan_smem_bytes(p, deck_smem);
    if (p.inside)
        return deck_smem ? dev::launch_t<true, true>(p, ctas, threads, smem, s)
                         : dev::launch_t<true, false>(p, ctas, threads, smem, s);
    return deck_smem ? dev::launch_t<false, true>(p, ctas, threads, smem, s)
                     : dev::launch_t<false, false>(p, ctas, threads, smem, s);
}

}  // namespace cmx
