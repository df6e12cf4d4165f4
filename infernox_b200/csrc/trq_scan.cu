// Truncated QDB / non-banded scan of whole windows (generic_tr_scan,
// src/cm_dpsearch_trunc.rs:1800-2316): ref_tr_cyk_scan (:207, f32 max-plus)
// and ref_itr_inside_scan (:226, i32 Inside with ILogsum).
//
// The reference's scan carries state from column to column beyond its
// rolling matrices: the ROOT row is never reset (a truncated begin competes
// with the best begin of every earlier column of the same parity), cells
// outside a state's band keep what an earlier column left there, and the
// BEGL decks are a ring over the last w+1 columns.  So one CTA runs one
// window, in HBM, on the reference's cell layout -- J/L/R/T planes of M
// state rows of w+1 cells per column, BEGL decks J/L/R of nbegl rows of w+1
// cells per column -- with the d = 0 cells set once when the window starts
// (the reference keeps two columns of planes and w+1 of BEGL decks; the
// column pipeline below keeps more, see there).  The states are
// grouped in dependency levels (one more than the deepest child; END states
// are level 0).  Every read of a cell (v, d) of the current column is of a
// lower level at d' <= d or of v's own cell d-1 (IL's self-loop); every read
// of an earlier column is of a lower level, or of v itself (IR), at d' <= d.
// So a column runs as a wavefront over (level, 8-cell chunk) -- unit (l, c)
// in step l + c, the truncated begins (ROOT) as the last level -- and
// column j+1 may run its step s as soon as column j has finished step s.
// A CTA's warps each run one column at a time (column jj on warp jj mod 8),
// step after step, waiting (on a shared-memory progress counter, with a
// bounded spin) only for the previous column's same step: no CTA-wide
// barriers, up to 8 columns of a window in flight.  The decks keep
// P = 9 column planes and a BEGL ring of w + 9 columns instead of the
// reference's 2 and w + 1; a warp starts column jj only after column jj-1
// began, hence after column jj-9 (the last one on that plane) and every
// reader of the ring slot it reuses have finished.  The values are the
// same: a state's band [1, dxcap] only grows with jrow, so a cell the
// reference reads from two columns back (its rolling matrices) was written
// in the previous column or never, and reads the same in any ring; the ROOT
// row, which the reference does carry across columns of the same parity,
// keeps two parities of its own.
// Plain cells take one lane each; an IL chunk of 8 cells is walked by one
// lane in d order, the self-transition value carried in a register,
// because the reference folds it second (after the local end value) and
// before the other children, an order Inside's rounding depends on.  Every
// cell folds its children in the reference's order with its comb (>= max
// for CYK, ILogsum for Inside), max2 (>= max) and wrapping i32 adds, so the
// results are the reference's bit for bit.  A ROOT cell d applies the
// truncated begins -- states ascending, planes J, L, R, then T for B
// states, the reference's order for one d -- to the persistent ROOT row,
// keeps the column's best begin and emits it if reportable; the host
// replays the greedy report with null3.  vsc_root is the first strict
// maximum in (j, d) order: each d keeps its best and the first column that
// reached it, reduced when the window ends.
//
// The CTAs are persistent: each owns one deck region and takes windows from
// a queue ordered longest first, so device memory is bounded by the resident
// CTAs and not by the batch.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "devbuf.h"
#include "model_internal.h"
#include "trunc_report.h"

namespace cmx {

struct TrqDev {
    int M = 0;
    int8_t *sttype = nullptr, *kind = nullptr;
    int32_t *cfirst = nullptr, *cnum = nullptr, *begl_idx = nullptr;
    uint32_t *tsc[2] = {nullptr, nullptr}, *esc[2] = {nullptr, nullptr}, *init_sc[2] = {nullptr, nullptr};
    std::vector<int> level, kind_h, begl_h;
    int nlev = 0, nbegl = 0;
    DevArena arena;
    int64_t cand_hint = 0;
    double last_ms = 0;
    int64_t last_cells = 0;
    int32_t last_launches = 0;
    int32_t stall_col = -1;  // test hook: this column never publishes its progress (next call only)
    int64_t deck_budget = (int64_t)4 << 30;  // bytes of decks resident at once (bounds the grid)
};

void trq_free(TrqDev *t) {
    if (!t) return;
    t->arena.release();
    cudaFree(t->sttype);
    cudaFree(t->kind);
    cudaFree(t->cfirst);
    cudaFree(t->cnum);
    cudaFree(t->begl_idx);
    for (int s = 0; s < 2; s++) {
        cudaFree(t->tsc[s]);
        cudaFree(t->esc[s]);
        cudaFree(t->init_sc[s]);
    }
    delete t;
}

namespace trq {

constexpr int THREADS = 256;
constexpr int NW = THREADS / 32;  // warps, columns in flight per window
constexpr int CH = 8;             // cells per wavefront unit
constexpr long long SPIN_LIMIT = 1ll << 24;  // polls of a wait (about a second) before it gives up
constexpr int END_E = 19;  // unique state id of END states (src/constants.rs)

// what a state does in the column loop
enum { K_SKIP = 0, K_B, K_BEGL, K_IL, K_ML, K_MRIR, K_MP, K_SD };

struct Win {
    int64_t dsq_off;
    int32_t i0, j0, w, idx;  // idx: the window's index in the caller's batch
};

struct Res {
    float vsc;
    int32_t vmode;
    float bsc_full;
    int32_t pad;
};

struct Tab {
    const int8_t *sttype, *kind;
    const int32_t *cfirst, *cnum, *dxcap, *begl_idx, *pbeg;
    const int32_t *cu_off, *il_off;  // [step][chunk 0..nc]: first unit of the step's chunk
    const int2 *units, *il_units;    // (state, first d) of 8-cell units, by (step, chunk)
    const uint32_t *tsc, *esc, *lm, *rm, *pty, *init_sc, *base;  // semiring words
    const uint16_t *ilog;
    int ilog_nz, M, W, nbegl, npbeg, nonbanded, fill_l, fill_r, fill_t;
    int nl, nc, nstep;  // levels, chunks, steps per column
    int stall_col;      // test hook (-1 off): the column whose warp never publishes
};

template <bool INS>
struct Sr;

template <>
struct Sr<false> {  // CYK: f32, ESL_MAX with >=
    typedef float T;
    __device__ static __forceinline__ T zero() { return -1.0e36f; }
    __device__ static __forceinline__ T add(T a, T b) { return __fadd_rn(a, b); }
    __device__ static __forceinline__ T comb(T a, T b, const uint16_t *, int) { return a >= b ? a : b; }
    __device__ static __forceinline__ T ld(const uint32_t *p) { return __uint_as_float(*p); }
    __device__ static __forceinline__ T tab(const uint32_t *p) { return __uint_as_float(__ldg(p)); }
    __device__ static __forceinline__ void st(uint32_t *p, T x) { *p = __float_as_uint(x); }
    __device__ static __forceinline__ float bits(T x) { return x; }
};

template <>
struct Sr<true> {  // Inside: i32 wrapping adds, ILogsum
    typedef int32_t T;
    __device__ static __forceinline__ T zero() { return -987654321; }
    __device__ static __forceinline__ T add(T a, T b) { return (int32_t)((uint32_t)a + (uint32_t)b); }
    // ILogsum (src/cp9.rs:65-75); the table is kept up to its last nonzero
    // entry nz, beyond which the rule adds 0
    __device__ static __forceinline__ T comb(T a, T b, const uint16_t *tbl, int nz) {
        int32_t mx = a > b ? a : b;
        if (mx < -987654321) mx = -987654321;
        const int32_t mn = a < b ? a : b;
        const uint32_t diff = (uint32_t)mx - (uint32_t)mn;
        if (mn <= -987654321 || diff >= (uint32_t)nz) return mx;
        return (int32_t)((uint32_t)mx + (uint32_t)tbl[diff]);
    }
    __device__ static __forceinline__ T ld(const uint32_t *p) { return (int32_t)*p; }
    __device__ static __forceinline__ T tab(const uint32_t *p) { return (int32_t)__ldg(p); }
    __device__ static __forceinline__ void st(uint32_t *p, T x) { *p = (uint32_t)x; }
    __device__ static __forceinline__ float bits(T x) {
        return x == -987654321 ? -1.0e36f : (float)((double)x / 1000.0);
    }
};

template <class T>
__device__ __forceinline__ T max2(T a, T b) {
    return a >= b ? a : b;
}

// one window's decks
struct Deck {
    uint32_t *J, *L, *R, *T, *BJ, *BL, *BR, *root;
    int W1, M, nbegl, RG;  // RG: BEGL ring length
    __device__ __forceinline__ uint32_t *c(uint32_t *P, int a, int v, int d) const {
        return P + ((size_t)(a * M + v) * W1 + d);
    }
    __device__ __forceinline__ uint32_t *b(uint32_t *P, int slot, int bi, int d) const {
        return P + ((size_t)(slot * nbegl + bi) * W1 + d);
    }
    // ROOT row of plane pl (J, L, R, T) for columns of parity par
    __device__ __forceinline__ uint32_t *rt(int pl, int par, int d) const {
        return root + ((size_t)(pl * 2 + par) * W1 + d);
    }
};

struct Col {
    int j, cur, prv, jrow, slot0;  // planes of columns j and j-1; slot0: BEGL ring slot of column j
    const uint8_t *dsq;
};

// cell (v, d) of every state kind but IL, as the reference computes it
template <bool INS>
__device__ __forceinline__ void cell(const Tab &t, const Deck &k, const Col &c, const uint16_t *lt, int v, int kind,
                                     int stt, int d) {
    using S = Sr<INS>;
    using T = typename S::T;
    const int nz = t.ilog_nz;
    const T Z = S::zero();
    const bool FL = t.fill_l, FR = t.fill_r, FT = t.fill_t;
    const uint32_t *isv = t.init_sc + (size_t)v * (t.W + 1);
    const uint32_t *ts = t.tsc + (size_t)v * MAXC;
    const uint32_t *esc = t.esc + (size_t)v * ESC;
    const int cur = c.cur, prv = c.prv;
    if (kind == K_B) {
        const int wl = t.cfirst[v], y = t.cnum[v], bi = t.begl_idx[wl];
        int kmin = 0, kmax = d;
        if (!t.nonbanded) {
            kmin = max(d - t.dxcap[wl], 0);
            kmax = min(t.dxcap[y], d);
        }
        const T a = S::tab(isv + d);
        T jsc = a, lsc = FL ? a : Z, rsc = FR ? a : Z, tsc2 = FT ? a : Z;
        // splits k ascending, BU at a time with their loads issued together;
        // the T plane (fill_t implies fill_l and fill_r) folds the same
        // loaded values over k = max(kmin,1)..min(d-1,kmax) in its own chain,
        // in the same ascending order as the reference's separate loop
        constexpr int BU = 8;
        for (int q0 = kmin; q0 <= kmax; q0 += BU) {
            T lj[BU], yj[BU], yl[BU], rb[BU];
#pragma unroll
            for (int u = 0; u < BU; u++) {
                const int q = min(q0 + u, kmax);
                int s = c.slot0 - q;
                if (s < 0) s += k.RG;
                lj[u] = S::ld(k.b(k.BJ, s, bi, d - q));
                yj[u] = S::ld(k.c(k.J, cur, y, q));
                yl[u] = FL ? S::ld(k.c(k.L, cur, y, q)) : Z;
                rb[u] = FR ? S::ld(k.b(k.BR, s, bi, d - q)) : Z;
            }
#pragma unroll
            for (int u = 0; u < BU; u++) {
                const int q = q0 + u;
                if (q <= kmax) {
                    jsc = S::comb(jsc, S::add(lj[u], yj[u]), lt, nz);
                    if (FL) lsc = S::comb(lsc, S::add(lj[u], yl[u]), lt, nz);
                    if (FR) rsc = S::comb(rsc, S::add(rb[u], yj[u]), lt, nz);
                    if (FT && q >= 1 && q <= d - 1) tsc2 = S::comb(tsc2, S::add(rb[u], yl[u]), lt, nz);
                }
            }
        }
        S::st(k.c(k.J, cur, v, d), jsc);
        if (FT) S::st(k.c(k.T, cur, v, d), tsc2);
        if (FL)
            S::st(k.c(k.L, cur, v, d),
                  kmin == 0 ? S::comb(lsc, max2(S::ld(k.b(k.BJ, c.slot0, bi, d)), S::ld(k.b(k.BL, c.slot0, bi, d))),
                                      lt, nz)
                            : lsc);
        if (FR)
            S::st(k.c(k.R, cur, v, d),
                  kmax == d ? S::comb(rsc, max2(S::ld(k.c(k.J, cur, y, d)), S::ld(k.c(k.R, cur, y, d))), lt, nz)
                            : rsc);
        return;
    }
    const int y = t.cfirst[v], cn = t.cnum[v];
    if (kind == K_BEGL || kind == K_SD) {  // S and D states: no emission, children at d
        const T a = S::tab(isv + d);
        T jsc = a, lsc = FL ? a : Z, rsc = FR ? a : Z;
        for (int yo = 0; yo < cn; yo++) {
            const T tv = S::tab(ts + yo);
            jsc = S::comb(jsc, S::add(S::ld(k.c(k.J, cur, y + yo, d)), tv), lt, nz);
            if (FL) lsc = S::comb(lsc, S::add(S::ld(k.c(k.L, cur, y + yo, d)), tv), lt, nz);
            if (FR) rsc = S::comb(rsc, S::add(S::ld(k.c(k.R, cur, y + yo, d)), tv), lt, nz);
        }
        if (kind == K_BEGL) {
            const int bi = t.begl_idx[v];
            S::st(k.b(k.BJ, c.slot0, bi, d), jsc);
            if (FL) S::st(k.b(k.BL, c.slot0, bi, d), lsc);
            if (FR) S::st(k.b(k.BR, c.slot0, bi, d), rsc);
        } else {
            S::st(k.c(k.J, cur, v, d), jsc);
            if (FL) S::st(k.c(k.L, cur, v, d), lsc);
            if (FR) S::st(k.c(k.R, cur, v, d), rsc);
        }
        return;
    }
    if (kind == K_ML) {  // left emitter without a self-loop
        const T a = S::tab(isv + d - 1);
        T jsc = a, lsc = FL ? a : Z;
        for (int yo = 0; yo < cn; yo++) {
            const T tv = S::tab(ts + yo);
            jsc = S::comb(jsc, S::add(S::ld(k.c(k.J, cur, y + yo, d - 1)), tv), lt, nz);
            if (FL) lsc = S::comb(lsc, S::add(S::ld(k.c(k.L, cur, y + yo, d - 1)), tv), lt, nz);
        }
        const T e = S::tab(esc + c.dsq[c.j - d + 1]);
        S::st(k.c(k.J, cur, v, d), S::add(jsc, e));
        if (FL) S::st(k.c(k.L, cur, v, d), d >= 2 ? S::add(lsc, e) : e);
        if (FR) {
            T rsc = S::tab(isv + d);
            for (int yo = 0; yo < cn; yo++) {
                const T tv = S::tab(ts + yo);
                rsc = S::comb(rsc,
                              max2(S::add(S::ld(k.c(k.J, cur, y + yo, d)), tv),
                                   S::add(S::ld(k.c(k.R, cur, y + yo, d)), tv)),
                              lt, nz);
            }
            S::st(k.c(k.R, cur, v, d), rsc);
        }
        return;
    }
    if (kind == K_MRIR) {  // right emitters: children one column back
        const T a = S::tab(isv + d - 1);
        T jsc = a, rsc = FR ? a : Z;
        for (int yo = 0; yo < cn; yo++) {
            const T tv = S::tab(ts + yo);
            jsc = S::comb(jsc, S::add(S::ld(k.c(k.J, prv, y + yo, d - 1)), tv), lt, nz);
            if (FR) rsc = S::comb(rsc, S::add(S::ld(k.c(k.R, prv, y + yo, d - 1)), tv), lt, nz);
        }
        const T ej = S::tab(esc + c.dsq[c.j]);
        S::st(k.c(k.J, cur, v, d), S::add(jsc, ej));
        if (FR) S::st(k.c(k.R, cur, v, d), d >= 2 ? S::add(rsc, ej) : ej);
        if (FL) {
            T lsc = S::tab(isv + d);
            for (int yo = stt == IR_ST ? 1 : 0; yo < cn; yo++) {
                const T tv = S::tab(ts + yo);
                lsc = S::comb(lsc,
                              max2(S::add(S::ld(k.c(k.J, cur, y + yo, d)), tv),
                                   S::add(S::ld(k.c(k.L, cur, y + yo, d)), tv)),
                              lt, nz);
            }
            S::st(k.c(k.L, cur, v, d), lsc);
        }
        return;
    }
    // K_MP
    const int xi = c.dsq[c.j - d + 1], xj = c.dsq[c.j];
    T jsc = d >= 2 ? S::tab(isv + d - 2) : Z;
    T lsc = FL ? S::tab(isv + d - 1) : Z, rsc = FR ? S::tab(isv + d - 1) : Z;
    for (int yo = 0; yo < cn; yo++) {
        const T tv = S::tab(ts + yo);
        if (d >= 2) jsc = S::comb(jsc, S::add(S::ld(k.c(k.J, prv, y + yo, d - 2)), tv), lt, nz);
        if (FL)
            lsc = S::comb(lsc,
                          max2(S::add(S::ld(k.c(k.J, cur, y + yo, d - 1)), tv),
                               S::add(S::ld(k.c(k.L, cur, y + yo, d - 1)), tv)),
                          lt, nz);
        if (FR)
            rsc = S::comb(rsc,
                          max2(S::add(S::ld(k.c(k.J, prv, y + yo, d - 1)), tv),
                               S::add(S::ld(k.c(k.R, prv, y + yo, d - 1)), tv)),
                          lt, nz);
    }
    S::st(k.c(k.J, cur, v, d), d >= 2 ? S::add(jsc, S::tab(esc + xi * KP + xj)) : Z);
    if (FL) {
        const T e = S::tab(t.lm + (size_t)v * KP + xi);
        S::st(k.c(k.L, cur, v, d), d >= 2 ? S::add(lsc, e) : e);
    }
    if (FR) {
        const T e = S::tab(t.rm + (size_t)v * KP + xj);
        S::st(k.c(k.R, cur, v, d), d >= 2 ? S::add(rsc, e) : e);
    }
}

// Cells d0..d1 of IL state v, in d order, by one lane: the self-transition
// value of cell d-1 is carried in a register (cell d0-1 comes from the
// previous step); the R plane reads only other children.
template <bool INS>
__device__ __forceinline__ void il_chunk(const Tab &t, const Deck &k, const Col &c, const uint16_t *lt, int v,
                                         int d0, int d1) {
    using S = Sr<INS>;
    using T = typename S::T;
    const int nz = t.ilog_nz;
    const T Z = S::zero();
    const bool FL = t.fill_l, FR = t.fill_r;
    const uint32_t *isv = t.init_sc + (size_t)v * (t.W + 1);
    const uint32_t *ts = t.tsc + (size_t)v * MAXC;
    const uint32_t *esc = t.esc + (size_t)v * ESC;
    const int cur = c.cur, y = t.cfirst[v], cn = t.cnum[v];
    T tv[MAXC];
#pragma unroll
    for (int yo = 0; yo < MAXC; yo++) tv[yo] = yo < cn ? S::tab(ts + yo) : Z;
    T carryJ = S::ld(k.c(k.J, cur, v, d0 - 1)), carryL = FL ? S::ld(k.c(k.L, cur, v, d0 - 1)) : Z;
#pragma unroll 1
    for (int d = d0; d <= d1; d++) {
        const T a = S::tab(isv + d - 1), e = S::tab(esc + c.dsq[c.j - d + 1]);
        T cj[MAXC], cl[MAXC];
#pragma unroll
        for (int yo = 0; yo < MAXC; yo++) {
            const bool other = yo < cn && y + yo != v;
            cj[yo] = other ? S::ld(k.c(k.J, cur, y + yo, d - 1)) : Z;
            cl[yo] = other && FL ? S::ld(k.c(k.L, cur, y + yo, d - 1)) : Z;
        }
        T jsc = a, lsc = FL ? a : Z;
#pragma unroll
        for (int yo = 0; yo < MAXC; yo++)
            if (yo < cn) {
                const bool self = y + yo == v;
                jsc = S::comb(jsc, S::add(self ? carryJ : cj[yo], tv[yo]), lt, nz);
                if (FL) lsc = S::comb(lsc, S::add(self ? carryL : cl[yo], tv[yo]), lt, nz);
            }
        carryJ = S::add(jsc, e);
        S::st(k.c(k.J, cur, v, d), carryJ);
        if (FL) {
            carryL = d >= 2 ? S::add(lsc, e) : e;
            S::st(k.c(k.L, cur, v, d), carryL);
        }
        if (FR) {
            T rsc = S::tab(isv + d);
#pragma unroll
            for (int yo = 1; yo < MAXC; yo++)
                if (yo < cn)
                    rsc = S::comb(rsc,
                                  max2(S::add(S::ld(k.c(k.J, cur, y + yo, d)), tv[yo]),
                                       S::add(S::ld(k.c(k.R, cur, y + yo, d)), tv[yo])),
                                  lt, nz);
            S::st(k.c(k.R, cur, v, d), rsc);
        }
    }
}

// ROOT cell d of a column: the truncated begins of the penalised states y
// (ascending) on planes J, L, R, then T (B states), into the ROOT row of the
// column's parity; the best begin of d is kept per d across columns and
// emitted if reportable.
template <bool INS>
__device__ __forceinline__ void root_cell(const Tab &t, const Deck &k, const Col &c, int d, float *vb, int *vbj,
                                          int *vbm, int j0, float *s_bsc, int widx, float cutoff, hb::TrCand *cand,
                                          int64_t cap, unsigned long long *ncand) {
    using S = Sr<INS>;
    using T = typename S::T;
    const T Z = S::zero();
    const bool FL = t.fill_l, FR = t.fill_r, FT = t.fill_t;
    const int par = c.j & 1;
    T rj = S::ld(k.rt(0, par, d)), rl = FL ? S::ld(k.rt(1, par, d)) : Z;
    T rr = FR ? S::ld(k.rt(2, par, d)) : Z, rt = FT ? S::ld(k.rt(3, par, d)) : Z;
    float bs = -1.0e36f;
    int bm = hb::TRM_UNKNOWN, br = 0;
    auto rec = [&](T sc, T &r, int mode, int y) {
        if (sc > r) {
            r = sc;
            const float f = S::bits(sc);
            if (f > bs) {
                bs = f;
                bm = mode;
                br = y;
            }
        }
    };
    // the begin states in order, RU at a time with their loads issued together
    constexpr int RU = 4;
    for (int q0 = 0; q0 < t.npbeg; q0 += RU) {
        T xj[RU], xl[RU], xr[RU], xt[RU];
        int yy[RU];
        bool ok[RU], okt[RU];
#pragma unroll
        for (int u = 0; u < RU; u++) {
            const int q = q0 + u;
            const int y = q < t.npbeg ? t.pbeg[q] : 0;
            yy[u] = y;
            ok[u] = q < t.npbeg && d <= t.dxcap[y];
            okt[u] = ok[u] && FT && t.sttype[y] == B_ST;
            const T pen = ok[u] ? S::tab(t.pty + y) : Z;
            xj[u] = ok[u] ? S::add(S::ld(k.c(k.J, c.cur, y, d)), pen) : Z;
            xl[u] = ok[u] && FL ? S::add(S::ld(k.c(k.L, c.cur, y, d)), pen) : Z;
            xr[u] = ok[u] && FR ? S::add(S::ld(k.c(k.R, c.cur, y, d)), pen) : Z;
            xt[u] = okt[u] ? S::add(S::ld(k.c(k.T, c.cur, y, d)), pen) : Z;
        }
#pragma unroll
        for (int u = 0; u < RU; u++) {
            if (!ok[u]) continue;
            rec(xj[u], rj, hb::TRM_J, yy[u]);
            if (FL) rec(xl[u], rl, hb::TRM_L, yy[u]);
            if (FR) rec(xr[u], rr, hb::TRM_R, yy[u]);
            if (okt[u]) rec(xt[u], rt, hb::TRM_T, yy[u]);
        }
    }
    S::st(k.rt(0, par, d), rj);
    if (FL) S::st(k.rt(1, par, d), rl);
    if (FR) S::st(k.rt(2, par, d), rr);
    if (FT) S::st(k.rt(3, par, d), rt);
    if (bs > vb[d]) {
        vb[d] = bs;
        vbj[d] = c.j;
        vbm[d] = bm;
    }
    if (c.j == j0 && d == j0) *s_bsc = bs;
    if (bs >= cutoff && bs > -1.0e36f) {
        const unsigned long long at = atomicAdd(ncand, 1ull);
        if ((int64_t)at < cap) cand[at] = hb::TrCand{widx, c.j, d, bs, bm, br};
    }
}

// Lane 0 polls a progress counter of another warp until it reaches `need`
// (or a wait of this CTA gave up, or SPIN_LIMIT polls pass: then it marks
// the error and gives up); the warp then sees every write that warp made
// before publishing.
__device__ __forceinline__ bool wait_for(volatile int *flag, int need, volatile int *err, int lane) {
    int ok = 1;
    if (lane == 0) {
        long long it = 0;
        while (*flag < need) {
            if (*err) {
                ok = 0;
                break;
            }
            if (++it > SPIN_LIMIT) {
                *err = 1;
                ok = 0;
                break;
            }
            __nanosleep(64);
        }
        __threadfence_block();
    }
    ok = __shfl_sync(0xffffffffu, ok, 0);
    __syncwarp();
    return ok;
}

// all of the warp's writes so far, then the new progress value
__device__ __forceinline__ void publish(volatile int *flag, int val, int lane) {
    __syncwarp();
    if (lane == 0) {
        __threadfence_block();
        *flag = val;
    }
    __syncwarp();
}

template <bool INS>
__global__ void __launch_bounds__(THREADS) trq_kernel(Tab t, const Win *__restrict__ wins, int nwin,
                                                      const uint8_t *__restrict__ dsq_all, uint32_t *decks,
                                                      int64_t deck_stride, float cutoff, int *queue, hb::TrCand *cand,
                                                      int64_t cap, unsigned long long *ncand, Res *res, int *kerr) {
    extern __shared__ __align__(16) unsigned char smem[];
    float *vb = (float *)smem;               // per d: best begin score over the columns so far
    int *vbj = (int *)(vb + t.W + 1);        // ... the first column that reached it
    int *vbm = vbj + t.W + 1;                // ... and its mode
    uint16_t *lt = (uint16_t *)(vbm + t.W + 1);
    __shared__ int s_win;
    __shared__ float s_bsc;
    __shared__ volatile int prog[NW];        // per warp: jj * S + steps done of its current column jj
    __shared__ volatile int s_err;
    const int tid = threadIdx.x, wid = tid >> 5, lane = tid & 31;
    if (INS)
        for (int x = tid; x < t.ilog_nz; x += THREADS) lt[x] = t.ilog[x];
    if (tid == 0) s_err = 0;
    const int M = t.M, nbegl = t.nbegl, P = NW + 1;
    const int S = t.nstep, NC = t.nc, NL = t.nl;
    uint32_t *dk = decks + (size_t)blockIdx.x * (size_t)deck_stride;
    for (;;) {
        __syncthreads();
        if (tid == 0) s_win = s_err ? nwin : atomicAdd(queue, 1);
        __syncthreads();
        const int wq = s_win;
        if (wq >= nwin) break;
        const Win wn = wins[wq];
        const int w = wn.w, W1 = w + 1, RG = W1 + NW;
        const size_t plane = (size_t)P * M * W1, bdeck = (size_t)RG * nbegl * W1;
        uint32_t *rbase = dk + 4 * plane, *bbase = rbase + 8 * (size_t)W1;
        const Deck k{dk, dk + plane, dk + 2 * plane, dk + 3 * plane, bbase, bbase + bdeck, bbase + 2 * bdeck, rbase,
                     W1, M, nbegl, RG};
        // every cell IMPOSSIBLE / -INFTY, then the d = 0 base cells
        const uint32_t zu = INS ? (uint32_t)(int32_t)-987654321 : __float_as_uint(-1.0e36f);
        for (size_t x = tid; x < 4 * plane + 8 * (size_t)W1; x += THREADS) {
            const int d = (int)(x % W1);
            const size_t r = x / W1;
            const int v = (int)(r % M), pl = (int)(r / ((size_t)P * M));
            dk[x] = (d == 0 && pl < 3 && x < 4 * plane) ? __ldg(t.base + (size_t)pl * M + v) : zu;
        }
        for (size_t x = tid; x < 3 * bdeck; x += THREADS) {
            const int d = (int)(x % W1);
            const int bi = (int)((x / W1) % nbegl);
            bbase[x] = (d == 0 && x < bdeck) ? __ldg(t.base + 3 * (size_t)M + bi) : zu;
        }
        for (int d = tid; d <= w; d += THREADS) {
            vb[d] = -1.0e36f;
            vbj[d] = 0;
            vbm[d] = hb::TRM_UNKNOWN;
        }
        if (tid < NW) prog[tid] = 0;
        if (tid == 0) s_bsc = -1.0e36f;
        __syncthreads();
        const uint8_t *dsq = dsq_all + wn.dsq_off;
        const int ncol = wn.j0 - wn.i0 + 1, dx0 = t.dxcap[0];
        bool ok = true;
        for (int jj = wid; jj < ncol && ok; jj += NW) {
            const int j = wn.i0 + jj, jrow = min(jj + 1, w);
            const Col c{j, j % P, (j - 1) % P, jrow, j % RG, dsq};
            const int ca = min((jrow + CH - 1) / CH, NC);
            for (int sp = 0; sp < S; sp++) {
                if (jj > 0 && !wait_for(&prog[(jj - 1) % NW], (jj - 1) * S + sp + 1, &s_err, lane)) {
                    ok = false;
                    break;
                }
                const int *ci = t.il_off + sp * (NC + 1), *cc = t.cu_off + sp * (NC + 1);
                // IL chunks, one lane each
                const int il0 = ci[0], nil = ci[ca] - il0;
                for (int x = lane; x < nil; x += 32) {
                    const int2 un = t.il_units[il0 + x];
                    const int d1 = min(min(jrow, t.dxcap[un.x]), un.y + CH - 1);
                    if (un.y <= d1) il_chunk<INS>(t, k, c, lt, un.x, un.y, d1);
                }
                // plain cells, then the ROOT cells of this step
                const int c0 = cc[0], ncu = cc[ca] - c0, rc = sp - NL;
                const bool root = rc >= 0 && rc * CH + 1 <= min(jrow, dx0);
                const int ntot = (ncu + (root ? 1 : 0)) * CH;
                for (int x = lane; x < ntot; x += 32) {
                    const int u = x / CH, m = x % CH;
                    if (u < ncu) {
                        const int2 un = t.units[c0 + u];
                        const int v = un.x, d = un.y + m;
                        if (d <= min(jrow, t.dxcap[v])) cell<INS>(t, k, c, lt, v, t.kind[v], t.sttype[v], d);
                    } else {
                        const int d = rc * CH + 1 + m;
                        if (d <= min(jrow, dx0))
                            root_cell<INS>(t, k, c, d, vb, vbj, vbm, wn.j0, &s_bsc, wn.idx, cutoff, cand, cap,
                                           ncand);
                    }
                }
                if (jj != t.stall_col)
                    publish(&prog[wid], jj * S + sp + 1, lane);
                else
                    __syncwarp();
            }
        }
        __syncthreads();
        if (tid == 0) {
            if (s_err) {
                atomicExch(kerr, 1);
            } else {
                float best = -1.0e36f;
                int bj = INT_MAX, bm = hb::TRM_UNKNOWN;
                for (int d = 1; d <= w; d++)
                    if (vb[d] > best || (vb[d] == best && best > -1.0e36f && vbj[d] < bj)) {
                        best = vb[d];
                        bj = vbj[d];
                        bm = vbm[d];
                    }
                res[wn.idx] = Res{best, bm, s_bsc, 0};
            }
        }
    }
}

}  // namespace trq

namespace {

#define TRQ_TRY(call)                                                                              \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess) {                                                                   \
            set_error(std::string("truncated QDB scan: ") + #call + ": " + cudaGetErrorString(e_)); \
            return CMGPU_EDEVICE;                                                                  \
        }                                                                                          \
    } while (0)

template <class T>
int upload_arr(T **dst, const T *src, size_t n) {
    if (cudaMalloc((void **)dst, std::max<size_t>(n, 1) * sizeof(T)) != cudaSuccess) return CMGPU_ENOMEM;
    if (n && cudaMemcpy(*dst, src, n * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess) return CMGPU_EDEVICE;
    return CMGPU_OK;
}

inline uint32_t fw(float x) {
    uint32_t u;
    std::memcpy(&u, &x, 4);
    return u;
}
inline uint32_t iw(int32_t x) { return (uint32_t)x; }

// the model's state kinds, dependency levels and BEGL deck indices
int trq_prepare(cmgpu_model *m, TrqDev **out) {
    std::lock_guard<std::mutex> g(m->mu);
    if (m->trq) {
        *out = m->trq;
        return CMGPU_OK;
    }
    const HostCM &c = m->cm;
    const int M = c.view.M;
    TrqDev *q = new TrqDev();
    q->M = M;
    q->level.assign(M, 0);
    q->kind_h.assign(M, trq::K_SKIP);
    q->begl_h.assign(M, -1);
    for (int v = 0; v < M; v++)
        if (c.stid[v] == BEGL_S) q->begl_h[v] = q->nbegl++;
    for (int v = M - 1; v >= 0; v--) {
        const int st = c.sttype[v];
        int l = 0;
        if (st == B_ST)
            l = 1 + std::max(q->level[c.cfirst[v]], q->level[c.cnum[v]]);
        else if (st != E_ST)
            for (int yo = 0; yo < c.cnum[v]; yo++) {
                const int y = c.cfirst[v] + yo;
                if (y != v) l = std::max(l, 1 + q->level[y]);
            }
        q->level[v] = l;
        if (v == 0 || st == E_ST) continue;
        const bool detached = v + 1 < M && c.stid[v + 1] == trq::END_E;
        int k = trq::K_SD;
        if (st == B_ST)
            k = trq::K_B;
        else if (c.stid[v] == BEGL_S)
            k = trq::K_BEGL;
        else if (st == IL_ST)
            k = detached ? trq::K_SKIP : trq::K_IL;
        else if (st == ML_ST)
            k = detached ? trq::K_SKIP : trq::K_ML;
        else if (st == MR_ST || st == IR_ST)
            k = detached ? trq::K_SKIP : trq::K_MRIR;
        else if (st == MP_ST)
            k = trq::K_MP;
        q->kind_h[v] = k;
        if (k != trq::K_SKIP) q->nlev = std::max(q->nlev, l + 1);
    }
    std::vector<int8_t> kind8(q->kind_h.begin(), q->kind_h.end());
    int rc = CMGPU_OK;
    if (cudaSetDevice(m->device) != cudaSuccess) rc = CMGPU_EDEVICE;
    if (!rc) rc = upload_arr(&q->sttype, c.sttype.data(), M);
    if (!rc) rc = upload_arr(&q->kind, kind8.data(), M);
    if (!rc) rc = upload_arr(&q->cfirst, c.cfirst.data(), M);
    if (!rc) rc = upload_arr(&q->cnum, c.cnum.data(), M);
    if (!rc) rc = upload_arr(&q->begl_idx, q->begl_h.data(), M);
    if (rc) {
        trq_free(q);
        set_error("truncated QDB scan: uploading the model tables failed");
        return rc;
    }
    m->trq = q;
    *out = q;
    return CMGPU_OK;
}

// per-semiring model tables: transitions, emissions and the local-end
// values init_sc[v][d] (built by repeated addition of the EL self score, as
// the reference builds them), uploaded on first use
int trq_semiring_tables(cmgpu_model *m, TrqDev *q, bool ins) {
    std::lock_guard<std::mutex> g(m->mu);
    const int s = ins ? 1 : 0;
    if (q->init_sc[s]) return CMGPU_OK;
    const HostCM &c = m->cm;
    const int M = c.view.M, W = c.view.W;
    std::vector<uint32_t> tsc((size_t)M * MAXC), esc((size_t)M * ESC), init((size_t)M * (W + 1));
    for (size_t x = 0; x < tsc.size(); x++) tsc[x] = ins ? iw(c.itsc[x]) : fw(c.tsc[x]);
    for (size_t x = 0; x < esc.size(); x++) esc[x] = ins ? iw(c.ioesc[x]) : fw(c.oesc[x]);
    if (ins) {
        std::vector<int32_t> el(W + 1);
        el[0] = 0;
        for (int d = 1; d <= W; d++) el[d] = (int32_t)((uint32_t)el[d - 1] + (uint32_t)c.view.iel_selfsc);
        for (int v = 0; v < M; v++)
            for (int d = 0; d <= W; d++)
                init[(size_t)v * (W + 1) + d] =
                    c.iendsc[v] == -INFTY ? iw(-INFTY) : iw((int32_t)((uint32_t)el[d] + (uint32_t)c.iendsc[v]));
    } else {
        std::vector<float> el(W + 1);
        el[0] = 0.0f;
        for (int d = 1; d <= W; d++) el[d] = el[d - 1] + c.view.el_selfsc;
        for (int v = 0; v < M; v++)
            for (int d = 0; d <= W; d++)
                init[(size_t)v * (W + 1) + d] =
                    !(c.endsc[v] > IMPOSSIBLE + 1.0f) ? fw(IMPOSSIBLE) : fw(el[d] + c.endsc[v]);
    }
    int rc = upload_arr(&q->tsc[s], tsc.data(), tsc.size());
    if (!rc) rc = upload_arr(&q->esc[s], esc.data(), esc.size());
    if (!rc) rc = upload_arr(&q->init_sc[s], init.data(), init.size());
    if (rc) set_error("truncated QDB scan: uploading the score tables failed");
    return rc;
}

// d = 0 cells set once per window (J, L, R planes [M] each, then the BEGL J
// deck per BEGL state), in the reference's order: states M-1 .. 0, a BEGL
// state before the B state that reads it
template <class T, class Add, class Max2>
void base_cells(const HostCM &c, const std::vector<int> &begl, int nbegl, const T *tsc, const T *endsc, T zero,
                T base0, Add add, Max2 mx2, std::vector<T> &out) {
    const int M = c.view.M;
    out.assign((size_t)3 * M + std::max(nbegl, 1), zero);
    T *bj = out.data(), *bl = bj + M, *br = bl + M, *bb = br + M;
    for (int v = M - 1; v >= 0; v--) {
        const int st = c.sttype[v];
        if (c.stid[v] != BEGL_S) {
            if (st == E_ST) {
                bj[v] = bl[v] = br[v] = base0;
            } else if (st == S_ST || st == D_ST) {
                T a0 = endsc[v];
                for (int yo = 0; yo < c.cnum[v]; yo++) a0 = mx2(a0, add(bj[c.cfirst[v] + yo], tsc[v * MAXC + yo]));
                bj[v] = mx2(a0, zero);
            } else if (st == B_ST) {
                bj[v] = add(bb[begl[c.cfirst[v]]], bj[c.cnum[v]]);
            }
        } else {
            T a0 = endsc[v];
            for (int yo = 0; yo < c.cnum[v]; yo++) a0 = mx2(a0, add(bj[c.cfirst[v] + yo], tsc[v * MAXC + yo]));
            bb[begl[v]] = mx2(a0, zero);
        }
    }
}

int trq_batch(const cmgpu_model *mc, cudaStream_t st, int semiring, int qdbidx, const cmgpu_tr_tables *tt,
              int pass_idx, int do_null3, const uint8_t *dsq_all, int64_t dsq_len, const cmgpu_window *wins,
              int32_t nwin, float cutoff, cmgpu_trq_result *results, std::vector<cmgpu_tr_hit> &hits) {
    cmgpu_model *m = const_cast<cmgpu_model *>(mc);
    const bool ins = semiring == CMGPU_INSIDE_I32;
    if (semiring != CMGPU_CYK_F32 && !ins) {
        set_error("truncated QDB scan: semiring must be CMGPU_CYK_F32 or CMGPU_INSIDE_I32");
        return CMGPU_EINVAL;
    }
    if (qdbidx < 0 || qdbidx > 2) {
        set_error("truncated QDB scan: qdbidx must be CMGPU_NOQDB, CMGPU_QDB1 or CMGPU_QDB2");
        return CMGPU_EINVAL;
    }
    if (!tt || !tt->lpos || !tt->rpos ||
        (ins ? (!tt->ilmesc || !tt->irmesc || !tt->ipty) : (!tt->lmesc || !tt->rmesc || !tt->pty))) {
        set_error("truncated QDB scan: missing truncation tables");
        return CMGPU_EINVAL;
    }
    // the truncated scanners take the truncated passes only: the reference
    // picks the pass's penalty row with pty_idx_for_pass(..).expect("truncated
    // pass") (src/cm_dpsearch_trunc.rs:219, src/cm_trunc.rs:99-107)
    if (pass_idx < 2 || pass_idx > 5) {
        set_error("truncated QDB scan: pass index must be a truncated pass 2..5 (PLI_PASS_*)");
        return CMGPU_EINVAL;
    }
    const HostCM &c = m->cm;
    const int M = c.view.M, W = c.view.W;
    for (int32_t e = 0; e < nwin; e++) {
        const cmgpu_window &wd = wins[e];
        if (wd.i0 < 1 || wd.dsq_offset < 0 || (wd.j0 >= wd.i0 && wd.dsq_offset + wd.j0 >= dsq_len)) {
            set_error("truncated QDB scan: window outside the residue buffer");
            return CMGPU_EINVAL;
        }
        if (wd.j0 >= wd.i0 && any_code_above_17(dsq_all + wd.dsq_offset + wd.i0, (int64_t)wd.j0 - wd.i0 + 1)) {
            set_error("truncated QDB scan: residue code above 17");
            return CMGPU_EINVAL;
        }
    }
    TrqDev *q = nullptr;
    int rc = trq_prepare(m, &q);
    if (!rc) rc = trq_semiring_tables(m, q, ins);
    if (rc) return rc;
    TRQ_TRY(cudaSetDevice(m->device));
    const int s = ins ? 1 : 0;
    // per-call tables: band caps, the level schedule's units, begins, bases
    std::vector<int32_t> dxcap(M);
    for (int v = 0; v < M; v++) {
        const int dmax = qdbidx == 0 ? W : (qdbidx == 1 ? c.dmax1[v] : c.dmax2[v]);
        dxcap[v] = std::min(dmax, W);
    }
    // the wavefront: unit (level l, chunk c) in step l + c over the levels
    // that hold work, the ROOT cells as one more level; a step's units sorted
    // by chunk (a column with fewer rows takes a prefix: cu_off / il_off),
    // then B units first and the rest by kind
    std::vector<int> lmap(std::max(q->nlev, 1), -1);
    for (int v = 1; v < M; v++)
        if (q->kind_h[v] != trq::K_SKIP && dxcap[v] >= 1) lmap[q->level[v]] = 0;
    int nl = 0;
    for (int &x : lmap)
        if (x == 0) x = nl++;
    const int NC = (W + trq::CH - 1) / trq::CH;
    const int nstep = nl + NC;
    struct U {
        int c, key, v, d0;
    };
    std::vector<std::vector<U>> sc_cells(nstep), sc_il(nstep);
    for (int v = 1; v < M; v++) {
        const int k = q->kind_h[v];
        if (k == trq::K_SKIP || dxcap[v] < 1) continue;
        for (int d0 = 1, ch = 0; d0 <= dxcap[v]; d0 += trq::CH, ch++) {
            const int sp = lmap[q->level[v]] + ch;
            (k == trq::K_IL ? sc_il : sc_cells)[sp].push_back(U{ch, k == trq::K_B ? 0 : k + 1, v, d0});
        }
    }
    std::vector<int2> units, il_units;
    std::vector<int32_t> cu_off((size_t)nstep * (NC + 1)), il_off((size_t)nstep * (NC + 1));
    auto lay = [&](std::vector<U> &L, std::vector<int2> &out, int32_t *off) {
        std::sort(L.begin(), L.end(), [](const U &a, const U &b) {
            if (a.c != b.c) return a.c < b.c;
            if (a.key != b.key) return a.key < b.key;
            if (a.v != b.v) return a.v < b.v;
            return a.d0 < b.d0;
        });
        size_t x = 0;
        for (int c = 0; c <= NC; c++) {
            while (x < L.size() && L[x].c < c) x++;
            off[c] = (int32_t)(out.size() + x);
        }
        for (const U &u : L) out.push_back(int2{u.v, u.d0});
    };
    for (int sp = 0; sp < nstep; sp++) {
        lay(sc_cells[sp], units, cu_off.data() + (size_t)sp * (NC + 1));
        lay(sc_il[sp], il_units, il_off.data() + (size_t)sp * (NC + 1));
    }
    std::vector<int32_t> pbeg;
    std::vector<uint32_t> lm((size_t)M * KP), rm((size_t)M * KP), pty(M), base;
    for (int y = 1; y < M; y++)
        if (ins ? tt->ipty[y] != -INFTY : tt->pty[y] > IMPOSSIBLE + 1.0f) pbeg.push_back(y);
    for (size_t x = 0; x < lm.size(); x++) {
        lm[x] = ins ? iw(tt->ilmesc[x]) : fw(tt->lmesc[x]);
        rm[x] = ins ? iw(tt->irmesc[x]) : fw(tt->rmesc[x]);
    }
    for (int v = 0; v < M; v++) pty[v] = ins ? iw(tt->ipty[v]) : fw(tt->pty[v]);
    if (ins) {
        std::vector<int32_t> b;
        base_cells<int32_t>(
            c, q->begl_h, q->nbegl, c.itsc.data(), c.iendsc.data(), -INFTY, 0,
            [](int32_t a, int32_t x) { return (int32_t)((uint32_t)a + (uint32_t)x); },
            [](int32_t a, int32_t x) { return a >= x ? a : x; }, b);
        for (int32_t x : b) base.push_back(iw(x));
    } else {
        std::vector<float> b;
        base_cells<float>(
            c, q->begl_h, q->nbegl, c.tsc.data(), c.endsc.data(), IMPOSSIBLE, 0.0f,
            [](float a, float x) { return a + x; }, [](float a, float x) { return a >= x ? a : x; }, b);
        for (float x : b) base.push_back(fw(x));
    }
    // windows: empty ones answer at once, the rest run longest first
    std::vector<trq::Win> wl;
    int wmax = 0;
    for (int32_t e = 0; e < nwin; e++) {
        const cmgpu_window &wd = wins[e];
        results[e] = cmgpu_trq_result{IMPOSSIBLE, hb::TRM_UNKNOWN, IMPOSSIBLE, 0, 0};
        if (wd.j0 < wd.i0) continue;
        const int L = wd.j0 - wd.i0 + 1, w = std::min(W, L);
        wl.push_back(trq::Win{wd.dsq_offset, wd.i0, wd.j0, w, e});
        wmax = std::max(wmax, w);
    }
    std::stable_sort(wl.begin(), wl.end(), [](const trq::Win &a, const trq::Win &b) {
        return (a.j0 - a.i0) > (b.j0 - b.i0);
    });
    // J-plane cells the scan computes, for the throughput counters
    std::vector<double> cnt(W + 1, 0.0);
    for (int r = 1; r <= W; r++)
        for (int v = 1; v < M; v++)
            if (q->kind_h[v] != trq::K_SKIP) cnt[r] += std::min(r, dxcap[v]);
    std::vector<double> pre(W + 1, 0.0);
    for (int r = 1; r <= W; r++) pre[r] = pre[r - 1] + cnt[r];
    double cells = 0;
    for (const trq::Win &x : wl) cells += pre[x.w] + (double)(x.j0 - x.i0 + 1 - x.w) * cnt[x.w];
    q->last_ms = 0;
    q->last_cells = (int64_t)cells;
    q->last_launches = 0;
    if (wl.empty()) return CMGPU_OK;

    const int nw = (int)wl.size();
    for (const trq::Win &x : wl)
        if ((int64_t)(x.j0 - x.i0 + 1) * nstep >= INT_MAX) {
            set_error("truncated QDB scan: window too long for the column progress counters");
            return CMGPU_EINVAL;
        }
    const int W1 = wmax + 1;
    const int nbk = std::max(q->nbegl, 1);  // the kernel's BEGL deck count (one unused deck without BEGL states)
    const int64_t nplane = trq::NW + 1;
    const int64_t deck_stride =
        ((int64_t)4 * nplane * M * W1 + (int64_t)8 * W1 + (int64_t)3 * (W1 + trq::NW) * nbk * W1 + 63) / 64 * 64;
    const size_t smem = (size_t)(W + 1) * 12 + (ins ? ((size_t)m->ilog_nz * 2 + 16) : 0);
    auto kfn = ins ? trq::trq_kernel<true> : trq::trq_kernel<false>;
    TRQ_TRY(cmx::allow_max_dynamic_smem(kfn));
    int occ = 0, nsm = 0;
    TRQ_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kfn, trq::THREADS, smem));
    TRQ_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, m->device));
    if (occ < 1) {
        set_error("truncated QDB scan: the kernel does not fit on an SM (W too large)");
        return CMGPU_EINVAL;
    }
    const int64_t budget = q->deck_budget;  // bytes of decks
    int64_t grid = std::min<int64_t>({(int64_t)nw, (int64_t)occ * nsm, std::max<int64_t>(1, budget / (deck_stride * 4))});

    DevArena &ar = q->arena;
    int2 *d_units, *d_il;
    int32_t *d_cuoff, *d_iloff, *d_dx, *d_pbeg;
    uint32_t *d_lm, *d_rm, *d_pty, *d_base, *d_decks;
    trq::Win *d_win;
    uint8_t *d_dsq;
    trq::Res *d_res;
    int *d_queue;
    unsigned long long *d_nc;
    if (ar.get(0, &d_units, sizeof(int2) * std::max<size_t>(units.size(), 1)) ||
        ar.get(1, &d_cuoff, sizeof(int32_t) * cu_off.size()) || ar.get(2, &d_dx, sizeof(int32_t) * M) ||
        ar.get(15, &d_il, sizeof(int2) * std::max<size_t>(il_units.size(), 1)) ||
        ar.get(16, &d_iloff, sizeof(int32_t) * il_off.size()) ||
        ar.get(3, &d_pbeg, sizeof(int32_t) * (pbeg.size() + 1)) || ar.get(4, &d_lm, sizeof(uint32_t) * lm.size()) ||
        ar.get(5, &d_rm, sizeof(uint32_t) * rm.size()) || ar.get(6, &d_pty, sizeof(uint32_t) * M) ||
        ar.get(7, &d_base, sizeof(uint32_t) * base.size()) || ar.get(8, &d_win, sizeof(trq::Win) * nw) ||
        ar.get(9, &d_dsq, (size_t)dsq_len) || ar.get(10, &d_res, sizeof(trq::Res) * nwin) ||
        ar.get(11, &d_decks, sizeof(uint32_t) * (size_t)deck_stride * (size_t)grid) ||
        ar.get(12, &d_queue, sizeof(int) * 2) || ar.get(13, &d_nc, sizeof(unsigned long long))) {
        set_error("truncated QDB scan: device allocation failed");
        return CMGPU_ENOMEM;
    }
    if (!units.empty())
        TRQ_TRY(cudaMemcpyAsync(d_units, units.data(), sizeof(int2) * units.size(), cudaMemcpyHostToDevice, st));
    if (!il_units.empty())
        TRQ_TRY(cudaMemcpyAsync(d_il, il_units.data(), sizeof(int2) * il_units.size(), cudaMemcpyHostToDevice, st));
    TRQ_TRY(cudaMemcpyAsync(d_cuoff, cu_off.data(), sizeof(int32_t) * cu_off.size(), cudaMemcpyHostToDevice, st));
    TRQ_TRY(cudaMemcpyAsync(d_iloff, il_off.data(), sizeof(int32_t) * il_off.size(), cudaMemcpyHostToDevice, st));
    TRQ_TRY(cudaMemcpyAsync(d_dx, dxcap.data(), sizeof(int32_t) * M, cudaMemcpyHostToDevice, st));
    if (!pbeg.empty())
        TRQ_TRY(cudaMemcpyAsync(d_pbeg, pbeg.data(), sizeof(int32_t) * pbeg.size(), cudaMemcpyHostToDevice, st));
    TRQ_TRY(cudaMemcpyAsync(d_lm, lm.data(), sizeof(uint32_t) * lm.size(), cudaMemcpyHostToDevice, st));
    TRQ_TRY(cudaMemcpyAsync(d_rm, rm.data(), sizeof(uint32_t) * rm.size(), cudaMemcpyHostToDevice, st));
    TRQ_TRY(cudaMemcpyAsync(d_pty, pty.data(), sizeof(uint32_t) * M, cudaMemcpyHostToDevice, st));
    TRQ_TRY(cudaMemcpyAsync(d_base, base.data(), sizeof(uint32_t) * base.size(), cudaMemcpyHostToDevice, st));
    TRQ_TRY(cudaMemcpyAsync(d_win, wl.data(), sizeof(trq::Win) * nw, cudaMemcpyHostToDevice, st));
    TRQ_TRY(cudaMemcpyAsync(d_dsq, dsq_all, (size_t)dsq_len, cudaMemcpyHostToDevice, st));
    const bool fill_l = pass_idx == 3 || pass_idx == 4 || pass_idx == 5;
    const bool fill_r = pass_idx == 2 || pass_idx == 4 || pass_idx == 5;
    const bool fill_t = pass_idx == 4 || pass_idx == 5;
    const trq::Tab tab{q->sttype, q->kind, q->cfirst, q->cnum, d_dx, q->begl_idx, d_pbeg, d_cuoff, d_iloff,
                       d_units, d_il, q->tsc[s], q->esc[s], d_lm, d_rm, d_pty, q->init_sc[s], d_base, m->ilog,
                       m->ilog_nz, M, W, nbk, (int)pbeg.size(), qdbidx == 0, fill_l, fill_r, fill_t,
                       nl, NC, nstep, q->stall_col};
    q->stall_col = -1;
    int64_t cap = std::max<int64_t>(4096 + 16 * (int64_t)nw, q->cand_hint);
    cudaEvent_t ev0, ev1;
    TRQ_TRY(cudaEventCreate(&ev0));
    TRQ_TRY(cudaEventCreate(&ev1));
    std::vector<hb::TrCand> hc;
    for (int attempt = 0; attempt < 2; attempt++) {
        hb::TrCand *d_c = nullptr;
        if (ar.get(14, &d_c, sizeof(hb::TrCand) * (size_t)cap)) {
            cudaEventDestroy(ev0);
            cudaEventDestroy(ev1);
            set_error("truncated QDB scan: device allocation failed");
            return CMGPU_ENOMEM;
        }
        TRQ_TRY(cudaMemsetAsync(d_queue, 0, sizeof(int) * 2, st));
        TRQ_TRY(cudaMemsetAsync(d_nc, 0, sizeof(unsigned long long), st));
        TRQ_TRY(cudaEventRecord(ev0, st));
        kfn<<<(unsigned)grid, trq::THREADS, smem, st>>>(tab, d_win, nw, d_dsq, d_decks, deck_stride, cutoff, d_queue,
                                                       d_c, cap, d_nc, d_res, d_queue + 1);
        TRQ_TRY(cudaGetLastError());
        TRQ_TRY(cudaEventRecord(ev1, st));
        unsigned long long nc = 0;
        int kerr = 0;
        TRQ_TRY(cudaMemcpyAsync(&nc, d_nc, sizeof(nc), cudaMemcpyDeviceToHost, st));
        TRQ_TRY(cudaMemcpyAsync(&kerr, d_queue + 1, sizeof(int), cudaMemcpyDeviceToHost, st));
        TRQ_TRY(cudaStreamSynchronize(st));
        if (kerr) {
            cudaEventDestroy(ev0);
            cudaEventDestroy(ev1);
            set_error("truncated QDB scan: a column wait of the kernel timed out");
            return CMGPU_ETIMEOUT;
        }
        float ms = 0;
        cudaEventElapsedTime(&ms, ev0, ev1);
        q->last_ms += ms;
        q->last_launches++;
        if ((int64_t)nc > cap) {
            cap = (int64_t)nc + (int64_t)nc / 4;
            q->cand_hint = cap;
            continue;
        }
        hc.resize((size_t)nc);
        if (nc)
            TRQ_TRY(cudaMemcpyAsync(hc.data(), d_c, sizeof(hb::TrCand) * (size_t)nc, cudaMemcpyDeviceToHost, st));
        break;
    }
    cudaEventDestroy(ev0);
    cudaEventDestroy(ev1);
    std::vector<trq::Res> rv(nwin);
    TRQ_TRY(cudaMemcpyAsync(rv.data(), d_res, sizeof(trq::Res) * nwin, cudaMemcpyDeviceToHost, st));
    TRQ_TRY(cudaStreamSynchronize(st));
    std::sort(hc.begin(), hc.end(), [](const hb::TrCand &a, const hb::TrCand &b) {
        if (a.env != b.env) return a.env < b.env;
        if (a.j != b.j) return a.j < b.j;
        return a.d < b.d;
    });
    const TrCtx cx{tt, pass_idx, tt->local};
    size_t p = 0;
    for (int32_t e = 0; e < nwin; e++) {
        const cmgpu_window &wd = wins[e];
        cmgpu_trq_result &r = results[e];
        r.hit_first = (int64_t)hits.size();
        size_t p1 = p;
        while (p1 < hc.size() && hc[p1].env == e) p1++;
        if (wd.j0 >= wd.i0) {
            r.vsc_root = rv[e].vsc;
            r.vmode = rv[e].vmode;
            r.bsc_full = rv[e].bsc_full;
            tr_report(m, cx, hc.data() + p, p1 - p, dsq_all + wd.dsq_offset, wd.i0, wd.j0, cutoff, do_null3, hits);
        }
        r.nhits = (int32_t)((int64_t)hits.size() - r.hit_first);
        p = p1;
    }
    return CMGPU_OK;
}

}  // namespace
}  // namespace cmx

using namespace cmx;

extern "C" int cmgpu_tr_qdb_scan_batch(const cmgpu_model *m, void *stream, int semiring, int qdbidx,
                                       const cmgpu_tr_tables *tt, int pass_idx, int do_null3, const uint8_t *dsq_all,
                                       int64_t dsq_len, const cmgpu_window *wins, int32_t nwin, float cutoff,
                                       cmgpu_trq_result *results, cmgpu_tr_hit *hits, int64_t cap, int64_t *n_out) {
    if (!m || !dsq_all || nwin < 0 || (nwin > 0 && (!wins || !results)) || !n_out) return CMGPU_EINVAL;
    *n_out = 0;
    if (nwin == 0) return CMGPU_OK;
    std::vector<cmgpu_tr_hit> all;
    int rc = trq_batch(m, (cudaStream_t)stream, semiring, qdbidx, tt, pass_idx, do_null3, dsq_all, dsq_len, wins,
                       nwin, cutoff, results, all);
    if (rc) return rc;
    *n_out = (int64_t)all.size();
    if ((int64_t)all.size() > cap) {
        set_error("cmgpu_tr_qdb_scan_batch: hit capacity too small");
        return CMGPU_EOVERFLOW;
    }
    if (hits) std::copy(all.begin(), all.end(), hits);
    return CMGPU_OK;
}

extern "C" int cmgpu_tr_qdb_scan(const cmgpu_model *m, int semiring, int qdbidx, const cmgpu_tr_tables *tt,
                                 const uint8_t *dsq, int32_t n, int32_t i0, int32_t j0, float cutoff, int do_null3,
                                 int pass_idx, float *vsc_root, int32_t *vmode, float *bsc_full, cmgpu_tr_hit *hits,
                                 int32_t cap, int32_t *n_out) {
    if (!m || !dsq || n < 0 || !vsc_root || !vmode || !bsc_full || !n_out) return CMGPU_EINVAL;
    *n_out = 0;
    if (j0 > n) {
        set_error("cmgpu_tr_qdb_scan: j0 beyond the sequence");
        return CMGPU_EINVAL;
    }
    const cmgpu_window wd{0, i0, j0};
    cmgpu_trq_result r{};
    std::vector<cmgpu_tr_hit> all;
    int rc = trq_batch(m, nullptr, semiring, qdbidx, tt, pass_idx, do_null3, dsq, (int64_t)n + 2, &wd, 1, cutoff, &r,
                       all);
    if (rc) return rc;
    *vsc_root = r.vsc_root;
    *vmode = r.vmode;
    *bsc_full = r.bsc_full;
    *n_out = (int32_t)all.size();
    if ((int64_t)all.size() > cap) {
        set_error("cmgpu_tr_qdb_scan: hit capacity too small");
        return CMGPU_EOVERFLOW;
    }
    if (hits) std::copy(all.begin(), all.end(), hits);
    return CMGPU_OK;
}

extern "C" int cmgpu_tr_qdb_inject_stall(cmgpu_model *m, int32_t column) {
    if (!m || column < -1) return CMGPU_EINVAL;
    TrqDev *q = nullptr;
    int rc = trq_prepare(m, &q);
    if (rc) return rc;
    q->stall_col = column;
    return CMGPU_OK;
}

extern "C" int cmgpu_tr_qdb_set_deck_budget(cmgpu_model *m, int64_t bytes) {
    if (!m || bytes < 0) return CMGPU_EINVAL;
    TrqDev *q = nullptr;
    int rc = trq_prepare(m, &q);
    if (rc) return rc;
    q->deck_budget = bytes > 0 ? bytes : ((int64_t)4 << 30);
    return CMGPU_OK;
}

extern "C" int cmgpu_tr_qdb_stats(const cmgpu_model *m, double *kernel_ms, int64_t *cells, int32_t *launches) {
    if (!m) return CMGPU_EINVAL;
    const TrqDev *q = m->trq;
    if (kernel_ms) *kernel_ms = q ? q->last_ms : 0.0;
    if (cells) *cells = q ? q->last_cells : 0;
    if (launches) *launches = q ? q->last_launches : 0;
    return CMGPU_OK;
}
