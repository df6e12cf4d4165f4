// HMM-banded (CP9-banded) CYK and float-Inside scans of envelopes
// (fast_cyk_scan_hb_core, src/cp9.rs:4717-5379; fast_finside_scan_hb,
// :5465-6014), many envelopes per launch, one CTA per envelope.
//
// Each envelope keeps the reference's banded matrix: state v, row jp = j -
// jmin[v], cells d = hdmin..hdmax stored contiguously from the row offset
// (in HBM; an envelope's working set stays in L2 while its states are
// computed).  The states are grouped in dependency levels on the host (a
// state's level is one more than its children's, END states are level 0), so
// every state of a level depends only on finished levels and itself.  A level
// is one phase of the CTA: its tasks are spread round-robin over the threads,
// a task being
//   * one band row (v, jp) for every state except IR -- its cells d run in
//     order in one thread, which is exactly what IL's self-transition (cell
//     d-1 of the same row) needs;
//   * one diagonal i = j-d+1 for IR states -- IR's self-transition reads
//     cell (j-1, d-1), the previous cell of the same diagonal, so the thread
//     walks the diagonal's rows in order.
// Every cell folds its children in the reference's order (children in
// ascending offset, bifurcation splits k ascending) starting from the local
// end value, then adds its emission and clamps at IMPOSSIBLE, so the float
// results are the reference's bit for bit (FLogsum is order-sensitive; MAX
// is taken with the reference's strict comparison).  After the last level a
// root pass applies the local begins (MAX in both semirings), finds vsc_root
// (first maximum in (j, d) order), the envelope of cells >= env_cutoff and the
// reportable cells; the host replays the greedy report with null3.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "devbuf.h"
#include "model_internal.h"
#include "trunc_report.h"

namespace cmx {

struct HbDev {
    int M = 0, nlev = 0, nbeg = 0;
    int8_t *sttype = nullptr;
    int32_t *cfirst = nullptr, *cnum = nullptr, *lev_start = nullptr, *lev_states = nullptr, *begins = nullptr;
    float *tsc = nullptr, *oesc = nullptr, *endsc = nullptr, *beginsc = nullptr, *flog = nullptr;
    double last_ms = 0;
    int64_t last_cells = 0;
    int32_t last_launches = 0;
    DevArena arena;          // per-call device buffers (tables, matrix, results), reused
    PinnedBuf st_pin, row_pin;  // per-call host band tables, staged in pinned memory
    int64_t cand_hint = 0;   // reportable cells the last call needed
    int64_t tr_cand_hint = 0;  // the same for the truncated scans
};

void hb_free(HbDev *h) {
    if (!h) return;
    h->arena.release();
    h->st_pin.release();
    h->row_pin.release();
    cudaFree(h->sttype);
    cudaFree(h->cfirst);
    cudaFree(h->cnum);
    cudaFree(h->lev_start);
    cudaFree(h->lev_states);
    cudaFree(h->begins);
    cudaFree(h->tsc);
    cudaFree(h->oesc);
    cudaFree(h->endsc);
    cudaFree(h->beginsc);
    cudaFree(h->flog);
    delete h;
}

namespace hb {

// threads per envelope CTA: one warp.  A dependency level rarely holds more
// than a few dozen band rows, a one-warp barrier is cheap, and sixteen
// envelopes share an SM (measured: 32 threads beat 64 by 20-34 %)
constexpr int HB_THREADS = 32;

struct Env {
    int64_t alpha_off;  // first cell of this envelope's matrix
    int64_t dsq_off;    // buffer index of residue 0
    int64_t row_off;    // first Row of this envelope
    int32_t i0, j0;
    float env_cutoff, cutoff;
    int32_t st_off;     // first State of this envelope
    int32_t pad;
};

struct State {
    int32_t jmin, jmax, row0, ntask;  // row0: first Row of state v within its envelope
    int32_t ilo, hmn_min, hmx_max, pad;  // IR: first diagonal, band extremes
};

struct Row {  // 8 bytes: band rows dominate the per-call copy
    int32_t roff;
    int16_t hmn, hmx;
};

struct Cand {
    int32_t env, j, d;
    float sc;
};

struct Out {
    float vsc;
    int32_t envi, envj, ncand;
};

struct Tables {
    const int8_t *sttype;
    const int32_t *cfirst, *cnum, *lev_start, *lev_states, *begins;
    const float *tsc, *oesc, *endsc, *beginsc, *flog;
    float el_selfsc;
    int nlev, nbeg, local_begin;
};

__device__ __forceinline__ int sdelta(int st) {
    return st == MP_ST ? 2 : (st == ML_ST || st == MR_ST || st == IL_ST || st == IR_ST) ? 1 : 0;
}
__device__ __forceinline__ int srdelta(int st) { return st == MP_ST || st == MR_ST || st == IR_ST; }

// FLogsum (src/cp9.rs:5405-5413)
__device__ __forceinline__ float flogsum(const float *tbl, float a, float b) {
    const float mx = fmaxf(a, b), mn = fminf(a, b);
    const float diff = __fsub_rn(mx, mn);
    if (mn == -INFINITY || diff >= 23.0f) return mx;
    return __fadd_rn(mx, __ldg(tbl + (int)__fmul_rn(diff, 1000.0f)));
}

template <bool INS>
__device__ __forceinline__ float comb(const float *tbl, float cur, float cand) {
    if (INS) return flogsum(tbl, cur, cand);
    return cand > cur ? cand : cur;
}

// Cells dlo..dhi of row jp of a non-bifurcation state v.
template <bool INS>
__device__ void row_cells(const Tables &t, const State *st, const Row *rows, float *alpha, const uint8_t *dsq,
                          int v, int stt, int jp, int dlo, int dhi) {
    const State sv = st[v];
    const int j = sv.jmin + jp;
    const Row rv = rows[sv.row0 + jp];
    const int av = rv.roff - rv.hmn;  // alpha[av + d] = cell d of this row
    const int sd = sdelta(stt), sdr = srdelta(stt);
    const float endsc = t.endsc[v];
    const bool has_end = endsc > -9.999e35f;
    if (stt == E_ST) {
        for (int d = dlo; d <= dhi; d++) {
            const float cur =
                has_end ? __fadd_rn(__fmul_rn(t.el_selfsc, (float)max(d - sd, 0)), endsc) : IMPOSSIBLE;
            alpha[av + d] = d == rv.hmn ? 0.0f : cur;
        }
        return;
    }
    const int ny = t.cnum[v], y0 = t.cfirst[v];
    int cx[MAXC], clo[MAXC], chi[MAXC];
    float ct[MAXC];
#pragma unroll
    for (int yo = 0; yo < MAXC; yo++) {
        clo[yo] = 1;
        chi[yo] = 0;
        cx[yo] = 0;
        ct[yo] = 0.0f;
        if (yo < ny) {
            const int y = y0 + yo, jy = j - sdr;
            const State sy = st[y];
            ct[yo] = t.tsc[v * MAXC + yo];
            if (jy >= sy.jmin && jy <= sy.jmax) {
                const Row ry = rows[sy.row0 + jy - sy.jmin];
                cx[yo] = ry.roff - ry.hmn - sd;  // alpha[cx + d] = child cell d - sd of row jy
                clo[yo] = ry.hmn + sd;
                chi[yo] = ry.hmx + sd;
            }
        }
    }
    const float *oesc = t.oesc + (size_t)v * ESC;
    const int xj = dsq[j];
    for (int d = dlo; d <= dhi; d++) {
        float cur = has_end ? __fadd_rn(__fmul_rn(t.el_selfsc, (float)max(d - sd, 0)), endsc) : IMPOSSIBLE;
#pragma unroll
        for (int yo = 0; yo < MAXC; yo++)
            if (d >= clo[yo] && d <= chi[yo]) cur = comb<INS>(t.flog, cur, __fadd_rn(alpha[cx[yo] + d], ct[yo]));
        if (stt == ML_ST || stt == IL_ST)
            cur = __fadd_rn(cur, oesc[dsq[j - d + 1]]);
        else if (stt == MR_ST || stt == IR_ST)
            cur = __fadd_rn(cur, oesc[xj]);
        else if (stt == MP_ST)
            cur = __fadd_rn(cur, oesc[dsq[j - d + 1] * KP + xj]);
        if (cur < IMPOSSIBLE) cur = IMPOSSIBLE;
        alpha[av + d] = cur;
    }
}

// Row jp of a bifurcation state v: split k over the right child z's row j.
template <bool INS>
__device__ void bif_row(const Tables &t, const State *st, const Row *rows, float *alpha, int v, int jp) {
    const State sv = st[v];
    const int j = sv.jmin + jp;
    const Row rv = rows[sv.row0 + jp];
    const int av = rv.roff - rv.hmn;
    const float endsc = t.endsc[v];
    const bool has_end = endsc > -9.999e35f;
    const int y = t.cfirst[v], z = t.cnum[v];
    const State sy = st[y], sz = st[z];
    const bool inz = j >= sz.jmin && j <= sz.jmax;
    Row rz{0, 1, 0};
    if (inz) rz = rows[sz.row0 + j - sz.jmin];
    const int jpy = j - sy.jmin;
    const int kn = max(max(j - sy.jmax, rz.hmn), 0), kx = min(jpy, rz.hmx);
    const int zx = rz.roff - rz.hmn;  // alpha[zx + k] = right child cell k
    for (int d = rv.hmn; d <= rv.hmx; d++) {
        float cur = has_end ? __fadd_rn(__fmul_rn(t.el_selfsc, (float)d), endsc) : IMPOSSIBLE;
        if (inz)
            for (int k = kn; k <= kx; k++) {
                const Row ry = rows[sy.row0 + jpy - k];
                if (k >= d - ry.hmx && k <= d - ry.hmn)
                    cur = comb<INS>(t.flog, cur, __fadd_rn(alpha[ry.roff + (d - ry.hmn - k)], alpha[zx + k]));
            }
        alpha[av + d] = cur;
    }
}

// IR state v, diagonal i: cells (j, j-i+1) in row order.
template <bool INS>
__device__ void ir_diag(const Tables &t, const State *st, const Row *rows, float *alpha, const uint8_t *dsq, int v,
                        int i) {
    const State sv = st[v];
    const int jlo = max(sv.jmin, i + sv.hmn_min - 1), jhi = min(sv.jmax, i + sv.hmx_max - 1);
    for (int j = jlo; j <= jhi; j++) {
        const int jp = j - sv.jmin, d = j - i + 1;
        const Row rv = rows[sv.row0 + jp];
        if (d >= rv.hmn && d <= rv.hmx) row_cells<INS>(t, st, rows, alpha, dsq, v, IR_ST, jp, d, d);
    }
}

template <bool INS>
__global__ void __launch_bounds__(HB_THREADS, 16) hb_kernel(Tables t, const Env *__restrict__ envs, int nenv,
                                                 const State *__restrict__ states, const Row *__restrict__ rows_all,
                                                 float *alpha_all, const uint8_t *__restrict__ dsq_all, int report,
                                                 Cand *cands, int64_t cand_cap, unsigned long long *ncand, Out *out) {
    __shared__ float s_v[HB_THREADS];
    __shared__ int s_j[HB_THREADS];
    __shared__ int s_envi, s_envj, s_nc;
    const int tid = threadIdx.x, nt = blockDim.x;
    for (int e = blockIdx.x; e < nenv; e += gridDim.x) {
        const Env env = envs[e];
        const State *st = states + env.st_off;
        const Row *rows = rows_all + env.row_off;
        float *alpha = alpha_all + env.alpha_off;
        const uint8_t *dsq = dsq_all + env.dsq_off;
        for (int lev = 0; lev < t.nlev; lev++) {
            int base = 0;
            for (int q = t.lev_start[lev]; q < t.lev_start[lev + 1]; q++) {
                const int v = t.lev_states[q];
                const int n = st[v].ntask, stt = t.sttype[v];
                // this thread's tasks: base + task = tid (mod nt)
                for (int task = ((tid - base) % nt + nt) % nt; task < n; task += nt) {
                    if (stt == IR_ST)
                        ir_diag<INS>(t, st, rows, alpha, dsq, v, st[v].ilo + task);
                    else if (stt == B_ST)
                        bif_row<INS>(t, st, rows, alpha, v, task);
                    else {
                        const Row r = rows[st[v].row0 + task];
                        if (r.hmn <= r.hmx) row_cells<INS>(t, st, rows, alpha, dsq, v, stt, task, r.hmn, r.hmx);
                    }
                }
                base += n;
            }
            __syncthreads();
        }
        // root pass: local begins, vsc_root, envelope, reportable cells
        if (tid == 0) {
            s_envi = INT_MAX;
            s_envj = INT_MIN;
            s_nc = 0;
        }
        __syncthreads();
        // vsc_root is the first maximum in (j, d) order: per row the first
        // strict maximum, per thread (rows ascending) a later row wins only
        // on a strictly larger value, across threads the smallest j wins ties
        float best = IMPOSSIBLE;
        int bestj = INT_MAX;
        const State s0 = st[0];
        for (int jp = tid; jp <= s0.jmax - s0.jmin; jp += nt) {
            const int j = s0.jmin + jp;
            const Row r0 = rows[s0.row0 + jp];
            const int av = r0.roff - r0.hmn;
            if (t.local_begin)
                for (int b = 0; b < t.nbeg; b++) {
                    const int y = t.begins[b];
                    const State sy = st[y];
                    if (j < sy.jmin || j > sy.jmax) continue;
                    const Row ry = rows[sy.row0 + j - sy.jmin];
                    const int dn = max(r0.hmn, ry.hmn), dx = min(r0.hmx, ry.hmx);
                    const float bsc = t.beginsc[y];
                    for (int d = dn; d <= dx; d++) {
                        const float sc = __fadd_rn(alpha[ry.roff + d - ry.hmn], bsc);
                        if (sc > alpha[av + d]) alpha[av + d] = sc;
                    }
                }
            float rb = IMPOSSIBLE;
            for (int d = r0.hmn; d <= r0.hmx; d++) {
                const float sc = alpha[av + d];
                if (sc > rb) rb = sc;
                if (sc >= env.env_cutoff) {
                    atomicMin(&s_envi, j - d + 1);
                    atomicMax(&s_envj, j);
                }
                if (report && d >= 1 && sc >= env.cutoff && sc > -9.999e35f) {
                    const unsigned long long slot = atomicAdd(ncand, 1ull);
                    atomicAdd(&s_nc, 1);
                    if ((int64_t)slot < cand_cap) cands[slot] = Cand{e, j, d, sc};
                }
            }
            if (rb > best) {
                best = rb;
                bestj = j;
            }
        }
        s_v[tid] = best;
        s_j[tid] = bestj;
        __syncthreads();
        if (tid == 0) {
            float bv = IMPOSSIBLE;
            int bj = INT_MAX;
            for (int q = 0; q < nt; q++)
                if (s_v[q] > bv || (s_v[q] == bv && s_j[q] < bj)) {
                    bv = s_v[q];
                    bj = s_j[q];
                }
            out[e] = Out{bv, s_envi == INT_MAX ? -1 : s_envi, s_envj == INT_MIN ? -1 : s_envj, s_nc};
        }
        __syncthreads();
    }
}


// ---------------------------------------------------------------------------
// Truncated scans (tr_cyk_scan_hb / ftr_inside_scan_hb): four planes J, L, R,
// T over the same banded layout (same cell index in each plane).  Each cell
// is computed plane by plane in the reference's order: the local-end value
// (planes with a left/right/no-emission offset), the children in ascending
// offset (J before L/R for one child), the emission rule of the state type,
// the IMPOSSIBLE clamp where the reference clamps; bifurcations fold splits k
// ascending, then the special L (left child only) and R (right child only)
// inherits.  ROOT is left out of the levels: its cells are the truncated
// begins, applied in the root pass.
// ---------------------------------------------------------------------------
struct TrTab {
    const float *lmesc, *rmesc, *pty;  // [M*18], [M*18], [M]
    const int32_t *pbeg;               // states y >= 1 with a truncated-begin penalty, ascending
    int npbeg, fill_l, fill_r, fill_t;
};

struct TrOut {
    float vsc;
    int32_t vmode, envi, envj;
};

struct CRow {
    int roff, hmn, hmx;
    bool ok;
};

__device__ __forceinline__ CRow crow(const State *st, const Row *rows, int y, int j) {
    const State sy = st[y];
    if (j < sy.jmin || j > sy.jmax) return CRow{0, 1, 0, false};
    const Row r = rows[sy.row0 + j - sy.jmin];
    return CRow{r.roff, r.hmn, r.hmx, true};
}

__device__ __forceinline__ int sldelta(int st) { return st == MP_ST || st == ML_ST || st == IL_ST; }

// plane validity of state y for this pass: bit 1 J, 2 L, 4 R, 8 T
__device__ __forceinline__ int tr_bits(const State *st, int y, const TrTab &tr) {
    const int b = st[y].pad;
    return (b & 1) | ((b & 2) && tr.fill_l ? 2 : 0) | ((b & 4) && tr.fill_r ? 4 : 0) | ((b & 8) && tr.fill_t ? 8 : 0);
}

// Cells dlo..dhi of row jp of a non-bifurcation state v (all four planes).
template <bool INS>
__device__ void tr_row(const Tables &t, const TrTab &tr, const State *st, const Row *rows, float *PJ, float *PL,
                       float *PR, float *PT, const uint8_t *dsq, int v, int stt, int jp, int dlo, int dhi) {
    const State sv = st[v];
    const int j = sv.jmin + jp;
    const Row rv = rows[sv.row0 + jp];
    const int base = rv.roff - rv.hmn;
    const int vb = tr_bits(st, v, tr);
    const bool dj = vb & 1, dl = vb & 2, dr = vb & 4;
    const int sd = sdelta(stt), sdl = sldelta(stt), sdr = srdelta(stt);
    const float endsc = t.endsc[v];
    const bool has_end = endsc > IMPOSSIBLE + 1.0f;
    auto init = [&](int d, int delta) -> float {
        return has_end && d >= delta ? __fadd_rn(__fmul_rn(t.el_selfsc, (float)(d - delta)), endsc) : IMPOSSIBLE;
    };
    if (stt == E_ST) {
        for (int d = dlo; d <= dhi; d++) {
            const int c = base + d;
            PJ[c] = dj ? (d == rv.hmn ? 0.0f : init(d, sd)) : IMPOSSIBLE;
            PL[c] = dl ? (d == rv.hmn ? 0.0f : init(d, sdl)) : IMPOSSIBLE;
            PR[c] = dr ? (d == rv.hmn ? 0.0f : init(d, sdr)) : IMPOSSIBLE;
            PT[c] = IMPOSSIBLE;
        }
        return;
    }
    const int ny = t.cnum[v], y0 = t.cfirst[v];
    CRow ca[MAXC], cb[MAXC];  // child rows at j - sdr and at j
    int cbits[MAXC];
    float ct[MAXC];
#pragma unroll
    for (int yo = 0; yo < MAXC; yo++) {
        ca[yo] = CRow{0, 1, 0, false};
        cb[yo] = ca[yo];
        cbits[yo] = 0;
        ct[yo] = 0.0f;
        if (yo < ny) {
            const int y = y0 + yo;
            ca[yo] = crow(st, rows, y, j - sdr);
            cb[yo] = sdr ? crow(st, rows, y, j) : ca[yo];
            cbits[yo] = tr_bits(st, y, tr);
            ct[yo] = t.tsc[v * MAXC + yo];
        }
    }
    const float *oesc = t.oesc + (size_t)v * ESC;
    const float *lm = tr.lmesc + (size_t)v * KP, *rm = tr.rmesc + (size_t)v * KP;
    const int xj = dsq[j];
    for (int d = dlo; d <= dhi; d++) {
        const int c = base + d;
        float J = dj ? init(d, sd) : IMPOSSIBLE, L = dl ? init(d, sdl) : IMPOSSIBLE, R = dr ? init(d, sdr) : IMPOSSIBLE;
        if (stt == ML_ST || stt == IL_ST) {
            const float e = oesc[dsq[j - d + 1]];
            if (dj || dl) {
#pragma unroll
                for (int yo = 0; yo < MAXC; yo++) {
                    const bool djy = cbits[yo] & 1, dly = cbits[yo] & 2;
                    if (!ca[yo].ok || !(djy || dly)) continue;
                    if (d - sd >= ca[yo].hmn && d - sd <= ca[yo].hmx) {
                        const int cy = ca[yo].roff + d - sd - ca[yo].hmn;
                        if (dj && djy) J = comb<INS>(t.flog, J, __fadd_rn(PJ[cy], ct[yo]));
                        if (dl && dly) L = comb<INS>(t.flog, L, __fadd_rn(PL[cy], ct[yo]));
                    }
                }
                if (dj) {
                    J = __fadd_rn(J, e);
                    if (J < IMPOSSIBLE) J = IMPOSSIBLE;
                }
                if (dl) {
                    L = d >= 2 ? __fadd_rn(L, e) : e;
                    if (L < IMPOSSIBLE) L = IMPOSSIBLE;
                }
            }
            if (dr) {
#pragma unroll
                for (int yo = 0; yo < MAXC; yo++) {
                    const bool djy = cbits[yo] & 1, dry = cbits[yo] & 4;
                    if (!ca[yo].ok || y0 + yo == v || !(djy || dry)) continue;
                    if (d >= ca[yo].hmn && d <= ca[yo].hmx) {
                        const int cy = ca[yo].roff + d - ca[yo].hmn;
                        if (djy) R = comb<INS>(t.flog, R, __fadd_rn(PJ[cy], ct[yo]));
                        if (dry) R = comb<INS>(t.flog, R, __fadd_rn(PR[cy], ct[yo]));
                    }
                }
            }
        } else if (stt == MR_ST || stt == IR_ST) {
            const float e = oesc[xj];
            if (dj || dr) {
#pragma unroll
                for (int yo = 0; yo < MAXC; yo++) {
                    const bool djy = cbits[yo] & 1, dry = cbits[yo] & 4;
                    if (!ca[yo].ok || !(djy || dry)) continue;
                    if (d - sd >= ca[yo].hmn && d - sd <= ca[yo].hmx) {
                        const int cy = ca[yo].roff + d - sd - ca[yo].hmn;
                        if (dj && djy) J = comb<INS>(t.flog, J, __fadd_rn(PJ[cy], ct[yo]));
                        if (dr && dry) R = comb<INS>(t.flog, R, __fadd_rn(PR[cy], ct[yo]));
                    }
                }
                if (dj) {
                    J = __fadd_rn(J, e);
                    if (J < IMPOSSIBLE) J = IMPOSSIBLE;
                }
                if (dr) {
                    R = d >= 2 ? __fadd_rn(R, e) : e;
                    if (R < IMPOSSIBLE) R = IMPOSSIBLE;
                }
            }
            if (dl) {
#pragma unroll
                for (int yo = 0; yo < MAXC; yo++) {
                    const bool djy = cbits[yo] & 1, dly = cbits[yo] & 2;
                    if (!cb[yo].ok || y0 + yo == v || !(djy || dly)) continue;
                    if (d >= cb[yo].hmn && d <= cb[yo].hmx) {
                        const int cy = cb[yo].roff + d - cb[yo].hmn;
                        if (djy) L = comb<INS>(t.flog, L, __fadd_rn(PJ[cy], ct[yo]));
                        if (dly) L = comb<INS>(t.flog, L, __fadd_rn(PL[cy], ct[yo]));
                    }
                }
            }
        } else if (stt == MP_ST) {
#pragma unroll
            for (int yo = 0; yo < MAXC; yo++) {
                if (yo >= ny) continue;
                const bool djy = cbits[yo] & 1, dly = cbits[yo] & 2, dry = cbits[yo] & 4;
                if (((dj && djy) || (dr && (djy || dry))) && ca[yo].ok) {
                    if (dj && djy && d - 2 >= ca[yo].hmn && d - 2 <= ca[yo].hmx)
                        J = comb<INS>(t.flog, J, __fadd_rn(PJ[ca[yo].roff + d - 2 - ca[yo].hmn], ct[yo]));
                    if (dr && (dry || djy) && d - 1 >= ca[yo].hmn && d - 1 <= ca[yo].hmx) {
                        const int cy = ca[yo].roff + d - 1 - ca[yo].hmn;
                        if (djy) R = comb<INS>(t.flog, R, __fadd_rn(PJ[cy], ct[yo]));
                        if (dry) R = comb<INS>(t.flog, R, __fadd_rn(PR[cy], ct[yo]));
                    }
                }
                if (dl && (dly || djy) && cb[yo].ok && d - 1 >= cb[yo].hmn && d - 1 <= cb[yo].hmx) {
                    const int cy = cb[yo].roff + d - 1 - cb[yo].hmn;
                    if (djy) L = comb<INS>(t.flog, L, __fadd_rn(PJ[cy], ct[yo]));
                    if (dly) L = comb<INS>(t.flog, L, __fadd_rn(PL[cy], ct[yo]));
                }
            }
            const int xi = dsq[j - d + 1];
            if (d >= 2) {
                if (dj) J = __fadd_rn(J, oesc[xi * KP + xj]);
                if (dl) L = __fadd_rn(L, lm[xi]);
                if (dr) R = __fadd_rn(R, rm[xj]);
            } else {
                if (dj) J = IMPOSSIBLE;
                if (dl) L = lm[xi];
                if (dr) R = rm[xj];
            }
            if (dj && J < IMPOSSIBLE) J = IMPOSSIBLE;
            if (dl && L < IMPOSSIBLE) L = IMPOSSIBLE;
            if (dr && R < IMPOSSIBLE) R = IMPOSSIBLE;
        } else {  // D, S: no emission, no clamp; L and R forced off at d = 0
#pragma unroll
            for (int yo = 0; yo < MAXC; yo++) {
                const bool djy = cbits[yo] & 1, dly = cbits[yo] & 2, dry = cbits[yo] & 4;
                if (!((dj && djy) || (dl && dly) || (dr && dry)) || !ca[yo].ok) continue;
                if (d - sd >= ca[yo].hmn && d - sd <= ca[yo].hmx) {
                    const int cy = ca[yo].roff + d - sd - ca[yo].hmn;
                    if (dj && djy) J = comb<INS>(t.flog, J, __fadd_rn(PJ[cy], ct[yo]));
                    if (dl && dly) L = comb<INS>(t.flog, L, __fadd_rn(PL[cy], ct[yo]));
                    if (dr && dry) R = comb<INS>(t.flog, R, __fadd_rn(PR[cy], ct[yo]));
                    if (d == 0) {
                        if (dl) L = IMPOSSIBLE;
                        if (dr) R = IMPOSSIBLE;
                    }
                }
            }
        }
        PJ[c] = J;
        PL[c] = L;
        PR[c] = R;
        PT[c] = IMPOSSIBLE;
    }
}

// Row jp of a bifurcation state v (all four planes).
template <bool INS>
__device__ void tr_bif_row(const Tables &t, const TrTab &tr, const State *st, const Row *rows, float *PJ, float *PL,
                           float *PR, float *PT, int v, int jp) {
    const State sv = st[v];
    const int j = sv.jmin + jp;
    const Row rv = rows[sv.row0 + jp];
    const int base = rv.roff - rv.hmn;
    const int vb = tr_bits(st, v, tr);
    const bool dj = vb & 1, dl = vb & 2, dr = vb & 4, dt = vb & 8;
    const float endsc = t.endsc[v];
    const bool has_end = endsc > IMPOSSIBLE + 1.0f;
    const int y = t.cfirst[v], z = t.cnum[v];
    const int yb = tr_bits(st, y, tr), zb = tr_bits(st, z, tr);
    const bool djy = yb & 1, dly = yb & 2, dry = yb & 4, djz = zb & 1, dlz = zb & 2, drz = zb & 4;
    const State sy = st[y];
    const CRow rz = crow(st, rows, z, j), ry = crow(st, rows, y, j);
    const int jpy = j - sy.jmin;
    const int kn = max(max(j - sy.jmax, rz.hmn), 0), kx = min(jpy, rz.hmx);
    for (int d = rv.hmn; d <= rv.hmx; d++) {
        const float e0 = has_end ? __fadd_rn(__fmul_rn(t.el_selfsc, (float)d), endsc) : IMPOSSIBLE;
        float J = dj ? e0 : IMPOSSIBLE, L = dl ? e0 : IMPOSSIBLE, R = dr ? e0 : IMPOSSIBLE, T = IMPOSSIBLE;
        if (rz.ok)
            for (int k = kn; k <= kx; k++) {
                const Row ryk = rows[sy.row0 + jpy - k];
                if (!(k >= d - ryk.hmx && k <= d - ryk.hmn)) continue;
                const int cy = ryk.roff + (d - ryk.hmn - k), cz = rz.roff + k - rz.hmn;
                if (dj && djy && djz) J = comb<INS>(t.flog, J, __fadd_rn(PJ[cy], PJ[cz]));
                if (dl && djy && dlz) L = comb<INS>(t.flog, L, __fadd_rn(PJ[cy], PL[cz]));
                if (dr && dry && djz) R = comb<INS>(t.flog, R, __fadd_rn(PR[cy], PJ[cz]));
                if (k != 0 && k != d && dt && dry && dlz) T = comb<INS>(t.flog, T, __fadd_rn(PR[cy], PL[cz]));
            }
        if (dl && (djy || dly) && ry.ok && d >= ry.hmn && d <= ry.hmx) {
            const int cy = ry.roff + d - ry.hmn;
            if (djy) L = comb<INS>(t.flog, L, PJ[cy]);
            if (dly) L = comb<INS>(t.flog, L, PL[cy]);
        }
        if (dr && (djz || drz) && rz.ok && d >= rz.hmn && d <= rz.hmx) {
            const int cz = rz.roff + d - rz.hmn;
            if (djz) R = comb<INS>(t.flog, R, PJ[cz]);
            if (drz) R = comb<INS>(t.flog, R, PR[cz]);
        }
        const int c = base + d;
        PJ[c] = J;
        PL[c] = L;
        PR[c] = R;
        PT[c] = T;
    }
}

template <bool INS>
__global__ void __launch_bounds__(HB_THREADS, 16) tr_kernel(Tables t, TrTab tr, const Env *__restrict__ envs, int nenv,
                                                 const State *__restrict__ states, const Row *__restrict__ rows_all,
                                                 float *planes, int64_t plane_stride, const uint8_t *__restrict__ dsq_all,
                                                 int report, TrCand *cands, int64_t cand_cap,
                                                 unsigned long long *ncand, TrOut *out) {
    __shared__ float s_v[HB_THREADS / 32];
    __shared__ int s_m[HB_THREADS / 32], s_j[HB_THREADS / 32];
    __shared__ int s_envi, s_envj;
    const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5, nwarp = nt >> 5;
    for (int e = blockIdx.x; e < nenv; e += gridDim.x) {
        const Env env = envs[e];
        const State *st = states + env.st_off;
        const Row *rows = rows_all + env.row_off;
        float *PJ = planes + env.alpha_off, *PL = PJ + plane_stride, *PR = PL + plane_stride, *PT = PR + plane_stride;
        const uint8_t *dsq = dsq_all + env.dsq_off;
        for (int lev = 0; lev < t.nlev; lev++) {
            int base = 0;
            for (int q = t.lev_start[lev]; q < t.lev_start[lev + 1]; q++) {
                const int v = t.lev_states[q];
                if (v == 0) continue;  // ROOT: truncated begins in the root pass
                const int n = st[v].ntask, stt = t.sttype[v];
                for (int task = ((tid - base) % nt + nt) % nt; task < n; task += nt) {
                    if (stt == IR_ST) {
                        const State sv = st[v];
                        const int i = sv.ilo + task;
                        const int jlo = max(sv.jmin, i + sv.hmn_min - 1), jhi = min(sv.jmax, i + sv.hmx_max - 1);
                        for (int j = jlo; j <= jhi; j++) {
                            const int d = j - i + 1;
                            const Row rv = rows[sv.row0 + j - sv.jmin];
                            if (d >= rv.hmn && d <= rv.hmx)
                                tr_row<INS>(t, tr, st, rows, PJ, PL, PR, PT, dsq, v, IR_ST, j - sv.jmin, d, d);
                        }
                    } else if (stt == B_ST) {
                        tr_bif_row<INS>(t, tr, st, rows, PJ, PL, PR, PT, v, task);
                    } else {
                        const Row r = rows[st[v].row0 + task];
                        if (r.hmn <= r.hmx) tr_row<INS>(t, tr, st, rows, PJ, PL, PR, PT, dsq, v, stt, task, r.hmn, r.hmx);
                    }
                }
                base += n;
            }
            __syncthreads();
        }
        // root pass: one warp per ROOT row, lanes over d.  Truncated begins
        // (MAX) into each plane with the best (score, mode, entry state) per
        // cell, then vsc_root -- the first maximum in (j, d, plane J/L/R/T)
        // order -- the envelope and the reportable cells.
        if (tid == 0) {
            s_envi = INT_MAX;
            s_envj = INT_MIN;
        }
        __syncthreads();
        const State s0 = st[0];
        const int b0 = tr_bits(st, 0, tr);
        float wbest = IMPOSSIBLE;
        int wmode = TRM_UNKNOWN, wj = INT_MAX;
        for (int jp = warp; jp <= s0.jmax - s0.jmin; jp += nwarp) {
            const int j = s0.jmin + jp;
            const Row r0 = rows[s0.row0 + jp];
            float rbest = IMPOSSIBLE;
            int rmode = TRM_UNKNOWN;
            for (int d0 = r0.hmn; d0 <= r0.hmx; d0 += 32) {
                const int d = d0 + lane;
                const bool act = d <= r0.hmx;
                float a[4] = {IMPOSSIBLE, IMPOSSIBLE, IMPOSSIBLE, IMPOSSIBLE};  // J L R T
                float best = IMPOSSIBLE;
                int bmode = TRM_UNKNOWN, broot = 0;
                for (int b = 0; b < tr.npbeg; b++) {
                    const int y = tr.pbeg[b];
                    const CRow ry = crow(st, rows, y, j);
                    if (!ry.ok || !act || d < ry.hmn || d > ry.hmx) continue;
                    const int yb = tr_bits(st, y, tr) & b0;
                    const float pen = tr.pty[y];
                    const int cy = ry.roff + d - ry.hmn;
                    const bool isb = t.sttype[y] == B_ST;
#pragma unroll
                    for (int pl = 0; pl < 4; pl++) {
                        if (!(yb & (1 << pl)) || (pl == 3 && !isb)) continue;
                        const float *P = pl == 0 ? PJ : pl == 1 ? PL : pl == 2 ? PR : PT;
                        const float sc = __fadd_rn(P[cy], pen);
                        if (sc > a[pl]) {
                            a[pl] = sc;
                            if (sc > best) {
                                best = sc;
                                bmode = pl == 0 ? TRM_J : pl == 1 ? TRM_L : pl == 2 ? TRM_R : TRM_T;
                                broot = y;
                            }
                        }
                    }
                }
                float cv = IMPOSSIBLE;
                int cmode = TRM_UNKNOWN;
                if (act) {
                    bool envhit = false;
#pragma unroll
                    for (int pl = 0; pl < 4; pl++) {
                        if (!(b0 & (1 << pl))) continue;
                        if (a[pl] > cv) {
                            cv = a[pl];
                            cmode = pl == 0 ? TRM_J : pl == 1 ? TRM_L : pl == 2 ? TRM_R : TRM_T;
                        }
                        if (a[pl] >= env.env_cutoff) envhit = true;
                    }
                    if (envhit) {
                        atomicMin(&s_envi, j - d + 1);
                        atomicMax(&s_envj, j);
                    }
                    if (report && d >= 1 && best >= env.cutoff && best > IMPOSSIBLE + 1.0f) {
                        const unsigned long long slot = atomicAdd(ncand, 1ull);
                        if ((int64_t)slot < cand_cap) cands[slot] = TrCand{e, j, d, best, bmode, broot};
                    }
                }
                // this chunk's first maximum (ties: smallest d); a later chunk
                // replaces the row's only with a strictly larger value
                float mx = cv;
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
                const unsigned at = __ballot_sync(0xffffffffu, act && cv == mx);
                const int first = __ffs(at) - 1;
                const int fmode = __shfl_sync(0xffffffffu, cmode, first < 0 ? 0 : first);
                if (first >= 0 && mx > rbest) {
                    rbest = mx;
                    rmode = fmode;
                }
            }
            if (rbest > wbest) {
                wbest = rbest;
                wmode = rmode;
                wj = j;
            }
        }
        if (lane == 0) {
            s_v[warp] = wbest;
            s_m[warp] = wmode;
            s_j[warp] = wj;
        }
        __syncthreads();
        if (tid == 0) {
            float bv = IMPOSSIBLE;
            int bm = TRM_UNKNOWN, bj = INT_MAX;
            for (int q = 0; q < nwarp; q++)
                if (s_v[q] > bv || (s_v[q] == bv && s_j[q] < bj)) {
                    bv = s_v[q];
                    bm = s_m[q];
                    bj = s_j[q];
                }
            out[e] = TrOut{bv, bm, s_envi == INT_MAX ? -1 : s_envi, s_envj == INT_MIN ? -1 : s_envj};
        }
        __syncthreads();
    }
}

}  // namespace hb

// ---------------------------------------------------------------------------
// truncated scans: host side
// ---------------------------------------------------------------------------
bool allow_trunc(const TrCtx &c, int64_t start, int64_t stop, int64_t i0, int64_t j0, int mode, int b) {
    if (c.pass_idx == 1 || c.pass_idx == 5) return true;  // STD_ANY, 5P_AND_3P_ANY
    if (start == i0 && stop == j0) return true;
    const int lp = c.tt->lpos[b], rp = c.tt->rpos[b];
    if (c.local) {
        if (mode == hb::TRM_J) return true;
        if (mode == hb::TRM_L) return stop == j0;
        if (mode == hb::TRM_R) return start == i0;
        return false;
    }
    if (mode == hb::TRM_J) return lp == 1 && rp == c.tt->clen;
    if (mode == hb::TRM_L) return stop == j0 && lp == 1;
    if (mode == hb::TRM_R) return start == i0 && rp == c.tt->clen;
    return false;
}

void tr_report(const cmgpu_model *m, const TrCtx &cx, const hb::TrCand *c, size_t n, const uint8_t *dsq, int32_t i0,
               int32_t j0, float cutoff, int do_null3, std::vector<cmgpu_tr_hit> &out) {
    std::vector<cmgpu_tr_hit> tmp;
    std::vector<int32_t> pre;
    const int32_t lo = i0 - 1;
    if (do_null3 && n) {
        const int32_t hi = c[n - 1].j;
        pre.assign((size_t)(hi - lo + 1) * 4, 0);
        for (int32_t p = lo + 1; p <= hi; p++) {
            for (int a = 0; a < 4; a++) pre[(size_t)(p - lo) * 4 + a] = pre[(size_t)(p - 1 - lo) * 4 + a];
            if (dsq[p] < 4) pre[(size_t)(p - lo) * 4 + dsq[p]]++;
        }
    }
    size_t k = 0;
    while (k < n) {
        const int32_t j = c[k].j;
        float max_rep = IMPOSSIBLE;
        for (; k < n && c[k].j == j; k++) {
            const int32_t d = c[k].d, i = j - d + 1;
            float sc = c[k].sc, bias = 0.0f;
            if (!(sc > max_rep && sc >= cutoff && sc > IMPOSSIBLE + 1.0f)) continue;
            bool rep = allow_trunc(cx, i, j, i0, j0, c[k].mode, c[k].root);
            if (rep && do_null3) {
                float comp[4], sum = 0.0f;
                for (int a = 0; a < 4; a++) {
                    comp[a] = (float)(double)(pre[(size_t)(j - lo) * 4 + a] - pre[(size_t)(i - 1 - lo) * 4 + a]);
                    sum += comp[a];
                }
                for (int a = 0; a < 4; a++) comp[a] = sum > 0.0f ? comp[a] / sum : 0.25f;
                const float corr = null3_corr(m, comp, d);
                sc -= corr;
                bias = corr;
                rep = sc > max_rep && sc >= cutoff;
            }
            if (rep) {
                tmp.push_back(cmgpu_tr_hit{i, j, sc, bias, c[k].mode, c[k].root});
                max_rep = sc;
            }
        }
    }
    std::stable_sort(tmp.begin(), tmp.end(), [](const cmgpu_tr_hit &a, const cmgpu_tr_hit &b) {
        if (a.score != b.score) return a.score > b.score;
        return a.i < b.i;
    });
    std::vector<char> removed(tmp.size(), 0);
    for (size_t a = 0; a < tmp.size(); a++) {
        if (removed[a]) continue;
        for (size_t b = a + 1; b < tmp.size(); b++)
            if (!removed[b] && !(tmp[b].j < tmp[a].i) && !(tmp[a].j < tmp[b].i)) removed[b] = 1;
    }
    for (size_t a = 0; a < tmp.size(); a++)
        if (!removed[a]) out.push_back(tmp[a]);
}

namespace {

template <class T>
int upload(T **dst, const T *src, size_t n) {
    if (cudaMalloc((void **)dst, std::max<size_t>(n, 1) * sizeof(T)) != cudaSuccess) return CMGPU_ENOMEM;
    if (n && cudaMemcpy(*dst, src, n * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess) return CMGPU_EDEVICE;
    return CMGPU_OK;
}

// model tables and the level schedule, built once per model
int hb_prepare(cmgpu_model *m, HbDev **out) {
    std::lock_guard<std::mutex> g(m->mu);
    if (m->hb) {
        *out = m->hb;
        return CMGPU_OK;
    }
    const HostCM &c = m->cm;
    const int M = c.view.M;
    std::vector<int> level(M, 0);
    int nlev = 0;
    for (int v = M - 1; v >= 0; v--) {
        const int st = c.sttype[v];
        int l = 0;
        if (st == B_ST)
            l = 1 + std::max(level[c.cfirst[v]], level[c.cnum[v]]);
        else if (st != E_ST)
            for (int yo = 0; yo < c.cnum[v]; yo++) {
                const int y = c.cfirst[v] + yo;
                if (y != v) l = std::max(l, 1 + level[y]);
            }
        level[v] = l;
        nlev = std::max(nlev, l + 1);
    }
    std::vector<int32_t> lev_start(nlev + 1, 0), lev_states(M);
    for (int v = 0; v < M; v++) lev_start[level[v] + 1]++;
    for (int l = 0; l < nlev; l++) lev_start[l + 1] += lev_start[l];
    std::vector<int32_t> fill(lev_start.begin(), lev_start.end() - 1);
    for (int v = M - 1; v >= 0; v--) lev_states[fill[level[v]]++] = v;
    std::vector<int32_t> begins;
    for (int y = 1; y < M; y++)
        if (c.beginsc[y] > -9.999e35f) begins.push_back(y);
    HbDev *h = new HbDev();
    h->M = M;
    h->nlev = nlev;
    h->nbeg = (int)begins.size();
    int rc = CMGPU_OK;
    if (cudaSetDevice(m->device) != cudaSuccess) rc = CMGPU_EDEVICE;
    if (!rc) rc = upload(&h->sttype, c.sttype.data(), M);
    if (!rc) rc = upload(&h->cfirst, c.cfirst.data(), M);
    if (!rc) rc = upload(&h->cnum, c.cnum.data(), M);
    if (!rc) rc = upload(&h->lev_start, lev_start.data(), lev_start.size());
    if (!rc) rc = upload(&h->lev_states, lev_states.data(), lev_states.size());
    if (!rc) rc = upload(&h->begins, begins.data(), begins.size());
    if (!rc) rc = upload(&h->tsc, c.tsc.data(), c.tsc.size());
    if (!rc) rc = upload(&h->oesc, c.oesc.data(), c.oesc.size());
    if (!rc) rc = upload(&h->endsc, c.endsc.data(), c.endsc.size());
    if (!rc) rc = upload(&h->beginsc, c.beginsc.data(), c.beginsc.size());
    if (!rc) rc = upload(&h->flog, m->flog.data(), m->flog.size());
    if (rc) {
        hb_free(h);
        set_error("HMM-banded scan: uploading the model tables failed");
        return rc;
    }
    m->hb = h;
    *out = h;
    return CMGPU_OK;
}

int sdelta_h(int st) { return st == MP_ST ? 2 : (st == ML_ST || st == MR_ST || st == IL_ST || st == IR_ST) ? 1 : 0; }

// rows of one envelope's bands (the sum of its states' j-ranges)
int64_t count_rows(int M, const cmgpu_hb_bands &b) {
    int64_t n = 0;
    for (int v = 0; v < M; v++) n += b.jmax[v] >= b.jmin[v] ? (int64_t)b.jmax[v] - b.jmin[v] + 1 : 0;
    return n;
}

// Validates one envelope's bands and fills its M States and its Rows (row
// indices and cell offsets relative to the envelope); returns the envelope's
// cell count, or -1 with err set.
int64_t fill_envelope(const HostCM &c, const cmgpu_hb_task &tk, int64_t dsq_len, const uint8_t *dsq_all,
                      hb::State *states, hb::Row *rows, std::string &err) {
    const int M = c.view.M;
    const cmgpu_hb_bands &b = tk.bands;
    if (tk.i0 < 1 || tk.j0 < tk.i0 - 1 || tk.dsq_offset < 0 || tk.dsq_offset + (int64_t)tk.j0 + 1 > dsq_len) {
        err = "HMM-banded scan: envelope outside the residue buffer";
        return -1;
    }
    if (tk.j0 >= tk.i0 && any_code_above_17(dsq_all + tk.dsq_offset + tk.i0, (int64_t)tk.j0 - tk.i0 + 1)) {
        err = "HMM-banded scan: residue code > 17";
        return -1;
    }
    int64_t ncells = 0;
    int32_t nrow = 0;
    for (int v = 0; v < M; v++) {
        const int st = c.sttype[v], sd = sdelta_h(st);
        hb::State s{b.jmin[v], b.jmax[v], nrow, 0, 0, INT_MAX, INT_MIN, 0};
        const int nj = b.jmax[v] >= b.jmin[v] ? b.jmax[v] - b.jmin[v] + 1 : 0;
        const int32_t *hmn_v = b.hdmin + b.hd_off[v], *hmx_v = b.hdmax + b.hd_off[v];
        int ilo = INT_MAX, ihi = INT_MIN;
        for (int jp = 0; jp < nj; jp++) {
            const int j = b.jmin[v] + jp, hmn = hmn_v[jp], hmx = hmx_v[jp];
            if (hmx >= hmn) {
                // every cell inside the envelope; emitting states need d >= 1
                // so that the residue(s) they emit lie inside it
                if (hmn < (sd > 0 ? 1 : 0) || j > tk.j0 || j - hmx + 1 < tk.i0) {
                    err = "HMM-banded scan: band cell outside the envelope (state " + std::to_string(v) + ", j " +
                          std::to_string(j) + ")";
                    return -1;
                }
                ilo = std::min(ilo, j - hmx + 1);
                ihi = std::max(ihi, j - hmn + 1);
                s.hmn_min = std::min(s.hmn_min, hmn);
                s.hmx_max = std::max(s.hmx_max, hmx);
            } else if (st == E_ST) {
                err = "HMM-banded scan: empty END state row";
                return -1;
            }
            if (hmn < -32768 || hmx > 32767) {
                err = "HMM-banded scan: band row beyond the 16-bit d range";
                return -1;
            }
            rows[nrow++] = hb::Row{(int32_t)ncells, (int16_t)hmn, (int16_t)hmx};
            if (hmx >= hmn) ncells += hmx - hmn + 1;
        }
        if (ncells > INT32_MAX) {
            err = "HMM-banded scan: more than 2^31 band cells in one envelope";
            return -1;
        }
        if (st == IR_ST) {
            s.ilo = ilo;
            s.ntask = ihi >= ilo ? ihi - ilo + 1 : 0;
        } else {
            s.ntask = nj;
        }
        states[v] = s;
    }
    return ncells;
}

// greedy report of one envelope from its reportable cells (sorted by j, d)
void hb_report(const cmgpu_model *m, const hb::Cand *c, size_t n, const uint8_t *dsq, int32_t i0, float cutoff,
               int do_null3, std::vector<cmgpu_hit> &out) {
    if (!n) return;
    std::vector<int32_t> pre;
    int32_t lo = i0 - 1, hi = c[n - 1].j;
    if (do_null3) {
        pre.assign((size_t)(hi - lo + 1) * 4, 0);
        for (int32_t p = lo + 1; p <= hi; p++) {
            for (int a = 0; a < 4; a++) pre[(size_t)(p - lo) * 4 + a] = pre[(size_t)(p - 1 - lo) * 4 + a];
            if (dsq[p] < 4) pre[(size_t)(p - lo) * 4 + dsq[p]]++;
        }
    }
    size_t k = 0;
    while (k < n) {
        const int32_t j = c[k].j;
        float max_rep = IMPOSSIBLE;
        for (; k < n && c[k].j == j; k++) {
            const int32_t d = c[k].d, i = j - d + 1;
            float hit_sc = c[k].sc, bias = 0.0f;
            if (!(hit_sc > max_rep && hit_sc >= cutoff && hit_sc > -9.999e35f)) continue;
            bool rep = true;
            if (do_null3) {
                float comp[4];
                for (int a = 0; a < 4; a++)
                    comp[a] = (float)(double)(pre[(size_t)(j - lo) * 4 + a] - pre[(size_t)(i - 1 - lo) * 4 + a]);
                // esl_vec_fnorm with a compensated sum (src/cp9.rs:464)
                float sum = 0.0f, cc = 0.0f;
                for (int a = 0; a < 4; a++) {
                    const float y = comp[a] - cc, t = sum + y;
                    cc = (t - sum) - y;
                    sum = t;
                }
                for (int a = 0; a < 4; a++) comp[a] = sum != 0.0f ? comp[a] / sum : 0.25f;
                const float corr = null3_corr(m, comp, d);
                hit_sc -= corr;
                bias = corr;
                rep = hit_sc > max_rep && hit_sc >= cutoff;
            }
            if (rep) {
                out.push_back(cmgpu_hit{i, j, hit_sc, bias});
                max_rep = hit_sc;
            }
        }
    }
}

#define HB_TRY(call)                                                                            \
    do {                                                                                        \
        cudaError_t e_ = (call);                                                                \
        if (e_ != cudaSuccess) {                                                                \
            set_error(std::string("HMM-banded scan: ") + #call + ": " + cudaGetErrorString(e_)); \
            return CMGPU_EDEVICE;                                                               \
        }                                                                                       \
    } while (0)

// one launch over envelopes [e0, e1), whose State and Row tables are staged
// in pinned memory (states: M per envelope; rows from row_base[e])
int hb_launch(cmgpu_model *m, HbDev *h, cudaStream_t st, int semiring, int report, int do_null3,
              const uint8_t *dsq_all, int64_t dsq_len, const cmgpu_hb_task *tasks, int32_t e0, int32_t e1,
              const hb::State *st_pin, const hb::Row *row_pin, const std::vector<int64_t> &row_base,
              const std::vector<int64_t> &alpha_off, cmgpu_hb_result *results, std::vector<cmgpu_hit> &hits,
              double &ms_total, int &launches) {
    const int n = e1 - e0;
    const int M = m->cm.view.M;
    const int64_t r0 = row_base[e0], nrows = row_base[e1] - r0;
    const int64_t cells = alpha_off[e1] - alpha_off[e0];
    std::vector<hb::Env> envs(n);
    for (int e = 0; e < n; e++) {
        const cmgpu_hb_task &tk = tasks[e0 + e];
        envs[e] = hb::Env{alpha_off[e0 + e] - alpha_off[e0], tk.dsq_offset, row_base[e0 + e] - r0, tk.i0, tk.j0,
                          tk.env_cutoff, tk.cutoff, e * M, 0};
    }
    hb::Env *d_env;
    hb::State *d_st;
    hb::Row *d_rows;
    float *d_alpha;
    uint8_t *d_dsq;
    hb::Out *d_out;
    unsigned long long *d_nc;
    DevArena &ar = h->arena;
    if (ar.get(0, &d_env, sizeof(hb::Env) * n) || ar.get(1, &d_st, sizeof(hb::State) * (size_t)n * M) ||
        ar.get(2, &d_rows, sizeof(hb::Row) * (size_t)nrows) || ar.get(3, &d_alpha, sizeof(float) * (size_t)cells) ||
        ar.get(4, &d_dsq, (size_t)dsq_len) || ar.get(5, &d_out, sizeof(hb::Out) * n) ||
        ar.get(6, &d_nc, sizeof(unsigned long long))) {
        set_error("HMM-banded scan: device allocation failed");
        return CMGPU_ENOMEM;
    }
    HB_TRY(cudaMemcpyAsync(d_env, envs.data(), sizeof(hb::Env) * n, cudaMemcpyHostToDevice, st));
    HB_TRY(cudaMemcpyAsync(d_st, st_pin + (size_t)e0 * M, sizeof(hb::State) * (size_t)n * M, cudaMemcpyHostToDevice,
                           st));
    HB_TRY(cudaMemcpyAsync(d_rows, row_pin + r0, sizeof(hb::Row) * (size_t)nrows, cudaMemcpyHostToDevice, st));
    HB_TRY(cudaMemcpyAsync(d_dsq, dsq_all, (size_t)dsq_len, cudaMemcpyHostToDevice, st));
    hb::Tables t{h->sttype, h->cfirst, h->cnum, h->lev_start, h->lev_states, h->begins, h->tsc, h->oesc,
                 h->endsc, h->beginsc, h->flog, m->cm.view.el_selfsc, h->nlev, h->nbeg,
                 (int)((m->cm.view.flags >> 10) & 1u)};
    int64_t cap = report ? std::max<int64_t>(4096 + 16 * (int64_t)n, h->cand_hint) : 0;
    cudaEvent_t ev0, ev1;
    HB_TRY(cudaEventCreate(&ev0));
    HB_TRY(cudaEventCreate(&ev1));
    for (int attempt = 0; attempt < 2; attempt++) {
        hb::Cand *d_c = nullptr;
        if (ar.get(7, &d_c, sizeof(hb::Cand) * (size_t)std::max<int64_t>(cap, 1))) {
            cudaEventDestroy(ev0);
            cudaEventDestroy(ev1);
            set_error("HMM-banded scan: device allocation failed");
            return CMGPU_ENOMEM;
        }
        HB_TRY(cudaMemsetAsync(d_nc, 0, sizeof(unsigned long long), st));
        HB_TRY(cudaEventRecord(ev0, st));
        if (semiring == CMGPU_INSIDE_F32)
            hb::hb_kernel<true><<<n, hb::HB_THREADS, 0, st>>>(t, d_env, n, d_st, d_rows, d_alpha, d_dsq, report, d_c, cap, d_nc,
                                                   d_out);
        else
            hb::hb_kernel<false><<<n, hb::HB_THREADS, 0, st>>>(t, d_env, n, d_st, d_rows, d_alpha, d_dsq, report, d_c, cap, d_nc,
                                                    d_out);
        HB_TRY(cudaGetLastError());
        HB_TRY(cudaEventRecord(ev1, st));
        unsigned long long nc = 0;
        std::vector<hb::Out> outv(n);
        HB_TRY(cudaMemcpyAsync(&nc, d_nc, sizeof(nc), cudaMemcpyDeviceToHost, st));
        HB_TRY(cudaMemcpyAsync(outv.data(), d_out, sizeof(hb::Out) * n, cudaMemcpyDeviceToHost, st));
        HB_TRY(cudaStreamSynchronize(st));
        float ms = 0;
        cudaEventElapsedTime(&ms, ev0, ev1);
        ms_total += ms;
        launches++;
        if ((int64_t)nc > cap) {
            cap = (int64_t)nc + (int64_t)nc / 4;
            h->cand_hint = cap;
            continue;
        }
        std::vector<hb::Cand> hc((size_t)nc);
        if (nc) {
            HB_TRY(cudaMemcpyAsync(hc.data(), d_c, sizeof(hb::Cand) * (size_t)nc, cudaMemcpyDeviceToHost, st));
            HB_TRY(cudaStreamSynchronize(st));
        }
        std::sort(hc.begin(), hc.end(), [](const hb::Cand &a, const hb::Cand &b) {
            if (a.env != b.env) return a.env < b.env;
            if (a.j != b.j) return a.j < b.j;
            return a.d < b.d;
        });
        size_t q = 0;
        for (int e = 0; e < n; e++) {
            const cmgpu_hb_task &tk = tasks[e0 + e];
            cmgpu_hb_result &r = results[e0 + e];
            r.vsc_root = outv[e].vsc;
            r.envi = outv[e].envi;
            r.envj = outv[e].envj;
            r.hit_first = (int64_t)hits.size();
            size_t q1 = q;
            while (q1 < hc.size() && hc[q1].env == e) q1++;
            if (report) hb_report(m, hc.data() + q, q1 - q, dsq_all + tk.dsq_offset, tk.i0, tk.cutoff, do_null3, hits);
            r.nhits = (int32_t)((int64_t)hits.size() - r.hit_first);
            q = q1;
        }
        break;
    }
    cudaEventDestroy(ev0);
    cudaEventDestroy(ev1);
    h->last_cells += cells;
    return CMGPU_OK;
}

int hb_batch(const cmgpu_model *mc, cudaStream_t st, int semiring, int report, int do_null3, const uint8_t *dsq_all,
             int64_t dsq_len, const cmgpu_hb_task *tasks, int32_t ntask, cmgpu_hb_result *results,
             std::vector<cmgpu_hit> &hits) {
    cmgpu_model *m = const_cast<cmgpu_model *>(mc);
    if (semiring != CMGPU_CYK_F32 && semiring != CMGPU_INSIDE_F32) {
        set_error("HMM-banded scan: semiring must be CMGPU_CYK_F32 or CMGPU_INSIDE_F32");
        return CMGPU_EINVAL;
    }
    for (int32_t e = 0; e < ntask; e++) {
        const cmgpu_hb_bands &b = tasks[e].bands;
        if (!b.jmin || !b.jmax || !b.hd_off || !b.hdmin || !b.hdmax) {
            set_error("HMM-banded scan: missing band arrays");
            return CMGPU_EINVAL;
        }
    }
    HbDev *h = nullptr;
    int rc = hb_prepare(m, &h);
    if (rc) return rc;
    HB_TRY(cudaSetDevice(m->device));
    const int M = m->cm.view.M;
    // band tables: count, then fill in parallel straight into pinned staging
    std::vector<int64_t> row_base(ntask + 1, 0), alpha_off(ntask + 1, 0), ncells(ntask, 0);
    for (int32_t e = 0; e < ntask; e++) row_base[e + 1] = row_base[e] + count_rows(M, tasks[e].bands);
    hb::State *st_pin = h->st_pin.get<hb::State>((size_t)ntask * M);
    hb::Row *row_pin = h->row_pin.get<hb::Row>((size_t)std::max<int64_t>(row_base[ntask], 1));
    if (!st_pin || !row_pin) {
        set_error("HMM-banded scan: pinned host allocation failed");
        return CMGPU_ENOMEM;
    }
    std::vector<std::string> errs(ntask);
    const int nthr = (int)std::max<int64_t>(1, std::min<int64_t>({(int64_t)std::thread::hardware_concurrency(), 32,
                                                                   (int64_t)ntask / 16 + 1}));
    auto work = [&](int32_t a, int32_t b) {
        for (int32_t e = a; e < b; e++)
            ncells[e] = fill_envelope(m->cm, tasks[e], dsq_len, dsq_all, st_pin + (size_t)e * M,
                                      row_pin + row_base[e], errs[e]);
    };
    if (nthr == 1) {
        work(0, ntask);
    } else {
        std::vector<std::thread> pool;
        for (int k = 0; k < nthr; k++)
            pool.emplace_back(work, (int32_t)((int64_t)ntask * k / nthr), (int32_t)((int64_t)ntask * (k + 1) / nthr));
        for (auto &t : pool) t.join();
    }
    for (int32_t e = 0; e < ntask; e++) {
        if (ncells[e] < 0) {
            set_error(errs[e]);
            return CMGPU_EINVAL;
        }
        alpha_off[e + 1] = alpha_off[e] + ncells[e];
    }
    h->last_ms = 0;
    h->last_cells = 0;
    h->last_launches = 0;
    // launches of at most ~1 Gi cells of matrix (4 GiB) each
    const int64_t budget = (int64_t)1 << 30;
    int launches = 0;
    double ms = 0;
    int32_t e0 = 0;
    while (e0 < ntask) {
        int32_t e1 = e0 + 1;
        while (e1 < ntask && alpha_off[e1 + 1] - alpha_off[e0] <= budget) e1++;
        rc = hb_launch(m, h, st, semiring, report, do_null3, dsq_all, dsq_len, tasks, e0, e1, st_pin, row_pin,
                       row_base, alpha_off, results, hits, ms, launches);
        if (rc) return rc;
        e0 = e1;
    }
    h->last_ms = ms;
    h->last_launches = launches;
    return CMGPU_OK;
}


int tr_launch(cmgpu_model *m, HbDev *h, cudaStream_t st, int semiring, const hb::TrTab &trt, const TrCtx &cx,
              int report, int do_null3, const uint8_t *dsq_all, int64_t dsq_len, const cmgpu_tr_task *tasks,
              int32_t e0, int32_t e1, const hb::State *st_pin, const hb::Row *row_pin,
              const std::vector<int64_t> &row_base, const std::vector<int64_t> &alpha_off,
              cmgpu_tr_result *results, std::vector<cmgpu_tr_hit> &hits, double &ms_total, int &launches) {
    const int n = e1 - e0;
    const int M = m->cm.view.M;
    const int64_t r0 = row_base[e0], nrows = row_base[e1] - r0;
    const int64_t cells = alpha_off[e1] - alpha_off[e0];
    std::vector<hb::Env> envs(n);
    for (int e = 0; e < n; e++) {
        const cmgpu_tr_task &tk = tasks[e0 + e];
        envs[e] = hb::Env{alpha_off[e0 + e] - alpha_off[e0], tk.dsq_offset, row_base[e0 + e] - r0, tk.i0, tk.j0,
                          tk.env_cutoff, tk.cutoff, e * M, 0};
    }
    hb::Env *d_env;
    hb::State *d_st;
    hb::Row *d_rows;
    float *d_planes;
    uint8_t *d_dsq;
    hb::TrOut *d_out;
    unsigned long long *d_nc;
    DevArena &ar = h->arena;
    if (ar.get(0, &d_env, sizeof(hb::Env) * n) || ar.get(1, &d_st, sizeof(hb::State) * (size_t)n * M) ||
        ar.get(2, &d_rows, sizeof(hb::Row) * (size_t)nrows) || ar.get(8, &d_planes, 4 * sizeof(float) * (size_t)cells) ||
        ar.get(4, &d_dsq, (size_t)dsq_len) || ar.get(10, &d_out, sizeof(hb::TrOut) * n) ||
        ar.get(6, &d_nc, sizeof(unsigned long long))) {
        set_error("truncated HMM-banded scan: device allocation failed");
        return CMGPU_ENOMEM;
    }
    HB_TRY(cudaMemcpyAsync(d_env, envs.data(), sizeof(hb::Env) * n, cudaMemcpyHostToDevice, st));
    HB_TRY(cudaMemcpyAsync(d_st, st_pin + (size_t)e0 * M, sizeof(hb::State) * (size_t)n * M, cudaMemcpyHostToDevice,
                           st));
    HB_TRY(cudaMemcpyAsync(d_rows, row_pin + r0, sizeof(hb::Row) * (size_t)nrows, cudaMemcpyHostToDevice, st));
    HB_TRY(cudaMemcpyAsync(d_dsq, dsq_all, (size_t)dsq_len, cudaMemcpyHostToDevice, st));
    hb::Tables t{h->sttype, h->cfirst, h->cnum, h->lev_start, h->lev_states, h->begins, h->tsc, h->oesc,
                 h->endsc, h->beginsc, h->flog, m->cm.view.el_selfsc, h->nlev, h->nbeg,
                 (int)((m->cm.view.flags >> 10) & 1u)};
    int64_t cap = report ? std::max<int64_t>(4096 + 16 * (int64_t)n, h->tr_cand_hint) : 0;
    cudaEvent_t ev0, ev1;
    HB_TRY(cudaEventCreate(&ev0));
    HB_TRY(cudaEventCreate(&ev1));
    for (int attempt = 0; attempt < 2; attempt++) {
        hb::TrCand *d_c = nullptr;
        if (ar.get(9, &d_c, sizeof(hb::TrCand) * (size_t)std::max<int64_t>(cap, 1))) {
            cudaEventDestroy(ev0);
            cudaEventDestroy(ev1);
            set_error("truncated HMM-banded scan: device allocation failed");
            return CMGPU_ENOMEM;
        }
        HB_TRY(cudaMemsetAsync(d_nc, 0, sizeof(unsigned long long), st));
        HB_TRY(cudaEventRecord(ev0, st));
        if (semiring == CMGPU_INSIDE_F32)
            hb::tr_kernel<true><<<n, hb::HB_THREADS, 0, st>>>(t, trt, d_env, n, d_st, d_rows, d_planes, cells, d_dsq, report, d_c,
                                                   cap, d_nc, d_out);
        else
            hb::tr_kernel<false><<<n, hb::HB_THREADS, 0, st>>>(t, trt, d_env, n, d_st, d_rows, d_planes, cells, d_dsq, report,
                                                    d_c, cap, d_nc, d_out);
        HB_TRY(cudaGetLastError());
        HB_TRY(cudaEventRecord(ev1, st));
        unsigned long long nc = 0;
        std::vector<hb::TrOut> outv(n);
        HB_TRY(cudaMemcpyAsync(&nc, d_nc, sizeof(nc), cudaMemcpyDeviceToHost, st));
        HB_TRY(cudaMemcpyAsync(outv.data(), d_out, sizeof(hb::TrOut) * n, cudaMemcpyDeviceToHost, st));
        HB_TRY(cudaStreamSynchronize(st));
        float ms = 0;
        cudaEventElapsedTime(&ms, ev0, ev1);
        ms_total += ms;
        launches++;
        if ((int64_t)nc > cap) {
            cap = (int64_t)nc + (int64_t)nc / 4;
            h->tr_cand_hint = cap;
            continue;
        }
        std::vector<hb::TrCand> hc((size_t)nc);
        if (nc) {
            HB_TRY(cudaMemcpyAsync(hc.data(), d_c, sizeof(hb::TrCand) * (size_t)nc, cudaMemcpyDeviceToHost, st));
            HB_TRY(cudaStreamSynchronize(st));
        }
        std::sort(hc.begin(), hc.end(), [](const hb::TrCand &a, const hb::TrCand &b) {
            if (a.env != b.env) return a.env < b.env;
            if (a.j != b.j) return a.j < b.j;
            return a.d < b.d;
        });
        size_t q = 0;
        for (int e = 0; e < n; e++) {
            const cmgpu_tr_task &tk = tasks[e0 + e];
            cmgpu_tr_result &r = results[e0 + e];
            r.vsc_root = outv[e].vsc;
            r.vmode = outv[e].vmode;
            r.envi = outv[e].envi;
            r.envj = outv[e].envj;
            r.hit_first = (int64_t)hits.size();
            size_t q1 = q;
            while (q1 < hc.size() && hc[q1].env == e) q1++;
            if (report)
                tr_report(m, cx, hc.data() + q, q1 - q, dsq_all + tk.dsq_offset, tk.i0, tk.j0, tk.cutoff, do_null3,
                          hits);
            r.nhits = (int32_t)((int64_t)hits.size() - r.hit_first);
            q = q1;
        }
        break;
    }
    cudaEventDestroy(ev0);
    cudaEventDestroy(ev1);
    h->last_cells += cells;
    return CMGPU_OK;
}

int tr_batch(const cmgpu_model *mc, cudaStream_t st, int semiring, const cmgpu_tr_tables *tt, int pass_idx,
             int report, int do_null3, const uint8_t *dsq_all, int64_t dsq_len, const cmgpu_tr_task *tasks,
             int32_t ntask, cmgpu_tr_result *results, std::vector<cmgpu_tr_hit> &hits) {
    cmgpu_model *m = const_cast<cmgpu_model *>(mc);
    if (semiring != CMGPU_CYK_F32 && semiring != CMGPU_INSIDE_F32) {
        set_error("truncated HMM-banded scan: semiring must be CMGPU_CYK_F32 or CMGPU_INSIDE_F32");
        return CMGPU_EINVAL;
    }
    if (!tt || !tt->lmesc || !tt->rmesc || !tt->pty || !tt->lpos || !tt->rpos) {
        set_error("truncated HMM-banded scan: missing truncation tables");
        return CMGPU_EINVAL;
    }
    // the truncated scanners take the truncated passes only: the reference
    // picks the pass's penalty row with pty_idx_for_pass(..).expect("truncated
    // pass") (src/cm_dpsearch_trunc.rs:219, src/cm_trunc.rs:99-107)
    if (pass_idx < 2 || pass_idx > 5) {
        set_error("truncated HMM-banded scan: pass index must be a truncated pass 2..5 (PLI_PASS_*)");
        return CMGPU_EINVAL;
    }
    for (int32_t e = 0; e < ntask; e++) {
        const cmgpu_tr_task &tk = tasks[e];
        if (!tk.bands.jmin || !tk.bands.jmax || !tk.bands.hd_off || !tk.bands.hdmin || !tk.bands.hdmax ||
            !tk.jvalid || !tk.lvalid || !tk.rvalid || !tk.tvalid) {
            set_error("truncated HMM-banded scan: missing band or validity arrays");
            return CMGPU_EINVAL;
        }
    }
    HbDev *h = nullptr;
    int rc = hb_prepare(m, &h);
    if (rc) return rc;
    HB_TRY(cudaSetDevice(m->device));
    const int M = m->cm.view.M;
    std::vector<int64_t> row_base(ntask + 1, 0), alpha_off(ntask + 1, 0), ncells(ntask, 0);
    for (int32_t e = 0; e < ntask; e++) row_base[e + 1] = row_base[e] + count_rows(M, tasks[e].bands);
    hb::State *st_pin = h->st_pin.get<hb::State>((size_t)std::max<int32_t>(ntask, 1) * M);
    hb::Row *row_pin = h->row_pin.get<hb::Row>((size_t)std::max<int64_t>(row_base[ntask], 1));
    if (!st_pin || !row_pin) {
        set_error("truncated HMM-banded scan: pinned host allocation failed");
        return CMGPU_ENOMEM;
    }
    std::vector<std::string> errs(ntask);
    const int nthr = (int)std::max<int64_t>(1, std::min<int64_t>({(int64_t)std::thread::hardware_concurrency(), 32,
                                                                   (int64_t)ntask / 16 + 1}));
    auto work = [&](int32_t a, int32_t b) {
        for (int32_t e = a; e < b; e++) {
            // the same band rules as the standard scan (cmgpu_hb_task shares the layout)
            const cmgpu_tr_task &tk = tasks[e];
            const cmgpu_hb_task ht{tk.dsq_offset, tk.i0, tk.j0, tk.env_cutoff, tk.cutoff, tk.bands};
            hb::State *sp = st_pin + (size_t)e * M;
            ncells[e] = fill_envelope(m->cm, ht, dsq_len, dsq_all, sp, row_pin + row_base[e], errs[e]);
            if (ncells[e] >= 0)
                for (int v = 0; v < M; v++)
                    sp[v].pad = (tk.jvalid[v] ? 1 : 0) | (tk.lvalid[v] ? 2 : 0) | (tk.rvalid[v] ? 4 : 0) |
                                (tk.tvalid[v] ? 8 : 0);
        }
    };
    if (nthr == 1) {
        work(0, ntask);
    } else {
        std::vector<std::thread> pool;
        for (int k = 0; k < nthr; k++)
            pool.emplace_back(work, (int32_t)((int64_t)ntask * k / nthr), (int32_t)((int64_t)ntask * (k + 1) / nthr));
        for (auto &th : pool) th.join();
    }
    for (int32_t e = 0; e < ntask; e++) {
        if (ncells[e] < 0) {
            set_error(errs[e]);
            return CMGPU_EINVAL;
        }
        alpha_off[e + 1] = alpha_off[e] + ncells[e];
    }
    // per-call tables: marginal emissions, penalties, the penalised states
    std::vector<int32_t> pbeg;
    for (int y = 1; y < M; y++)
        if (tt->pty[y] > IMPOSSIBLE + 1.0f) pbeg.push_back(y);
    float *d_lm, *d_rm, *d_pty;
    int32_t *d_pbeg;
    DevArena &ar = h->arena;
    if (ar.get(11, &d_lm, sizeof(float) * (size_t)M * KP) || ar.get(12, &d_rm, sizeof(float) * (size_t)M * KP) ||
        ar.get(13, &d_pty, sizeof(float) * (size_t)M) || ar.get(14, &d_pbeg, sizeof(int32_t) * (pbeg.size() + 1))) {
        set_error("truncated HMM-banded scan: device allocation failed");
        return CMGPU_ENOMEM;
    }
    HB_TRY(cudaMemcpyAsync(d_lm, tt->lmesc, sizeof(float) * (size_t)M * KP, cudaMemcpyHostToDevice, st));
    HB_TRY(cudaMemcpyAsync(d_rm, tt->rmesc, sizeof(float) * (size_t)M * KP, cudaMemcpyHostToDevice, st));
    HB_TRY(cudaMemcpyAsync(d_pty, tt->pty, sizeof(float) * (size_t)M, cudaMemcpyHostToDevice, st));
    if (!pbeg.empty())
        HB_TRY(cudaMemcpyAsync(d_pbeg, pbeg.data(), sizeof(int32_t) * pbeg.size(), cudaMemcpyHostToDevice, st));
    const bool fill_l = pass_idx == 3 || pass_idx == 4 || pass_idx == 5;
    const bool fill_r = pass_idx == 2 || pass_idx == 4 || pass_idx == 5;
    const bool fill_t = pass_idx == 4 || pass_idx == 5;
    const hb::TrTab trt{d_lm, d_rm, d_pty, d_pbeg, (int)pbeg.size(), fill_l, fill_r, fill_t};
    const TrCtx cx{tt, pass_idx, tt->local};
    h->last_ms = 0;
    h->last_cells = 0;
    h->last_launches = 0;
    const int64_t budget = (int64_t)1 << 28;  // cells per launch (four planes: 4 GiB)
    int launches = 0;
    double ms = 0;
    int32_t e0 = 0;
    while (e0 < ntask) {
        int32_t e1 = e0 + 1;
        while (e1 < ntask && alpha_off[e1 + 1] - alpha_off[e0] <= budget) e1++;
        rc = tr_launch(m, h, st, semiring, trt, cx, report, do_null3, dsq_all, dsq_len, tasks, e0, e1, st_pin,
                       row_pin, row_base, alpha_off, results, hits, ms, launches);
        if (rc) return rc;
        e0 = e1;
    }
    h->last_ms = ms;
    h->last_launches = launches;
    return CMGPU_OK;
}

}  // namespace
}  // namespace cmx

using namespace cmx;

extern "C" int cmgpu_hb_scan_batch(const cmgpu_model *m, void *stream, int semiring, int report_hits, int do_null3,
                                   const uint8_t *dsq_all, int64_t dsq_len, const cmgpu_hb_task *tasks,
                                   int32_t ntask, cmgpu_hb_result *results, cmgpu_hit *hits, int64_t cap,
                                   int64_t *n_out) {
    if (!m || !dsq_all || ntask < 0 || (ntask > 0 && (!tasks || !results)) || !n_out) return CMGPU_EINVAL;
    *n_out = 0;
    if (ntask == 0) return CMGPU_OK;
    std::vector<cmgpu_hit> all;
    int rc = hb_batch(m, (cudaStream_t)stream, semiring, report_hits, do_null3, dsq_all, dsq_len, tasks, ntask,
                      results, all);
    if (rc) return rc;
    *n_out = (int64_t)all.size();
    if ((int64_t)all.size() > cap) {
        set_error("cmgpu_hb_scan_batch: hit capacity too small");
        return CMGPU_EOVERFLOW;
    }
    if (hits) std::copy(all.begin(), all.end(), hits);
    return CMGPU_OK;
}

extern "C" int cmgpu_fast_cyk_scan_hb(const cmgpu_model *m, const cmgpu_hb_bands *bands, const uint8_t *dsq,
                                      int32_t n, int32_t i0, int32_t j0, float env_cutoff, float *vsc_root,
                                      int64_t *envi, int64_t *envj) {
    if (!m || !bands || !dsq || n < 0 || !vsc_root || !envi || !envj) return CMGPU_EINVAL;
    cmgpu_hb_task tk{0, i0, j0, env_cutoff, 0.0f, *bands};
    cmgpu_hb_result r{};
    std::vector<cmgpu_hit> hits;
    int rc = hb_batch(m, nullptr, CMGPU_CYK_F32, 0, 0, dsq, (int64_t)n + 2, &tk, 1, &r, hits);
    if (rc) return rc;
    *vsc_root = r.vsc_root;
    *envi = r.envi;
    *envj = r.envj;
    return CMGPU_OK;
}

extern "C" int cmgpu_hb_scan_hits(const cmgpu_model *m, int semiring, const cmgpu_hb_bands *bands,
                                  const uint8_t *dsq, int32_t n, int32_t i0, int32_t j0, float env_cutoff,
                                  float cutoff, int do_null3, float *vsc_root, int64_t *envi, int64_t *envj,
                                  cmgpu_hit *hits, int32_t cap, int32_t *n_out) {
    if (!m || !bands || !dsq || n < 0 || !vsc_root || !envi || !envj || !n_out) return CMGPU_EINVAL;
    *n_out = 0;
    cmgpu_hb_task tk{0, i0, j0, env_cutoff, cutoff, *bands};
    cmgpu_hb_result r{};
    std::vector<cmgpu_hit> all;
    int rc = hb_batch(m, nullptr, semiring, 1, do_null3, dsq, (int64_t)n + 2, &tk, 1, &r, all);
    if (rc) return rc;
    *vsc_root = r.vsc_root;
    *envi = r.envi;
    *envj = r.envj;
    *n_out = (int32_t)all.size();
    if ((int64_t)all.size() > cap) {
        set_error("cmgpu_hb_scan_hits: hit capacity too small");
        return CMGPU_EOVERFLOW;
    }
    if (hits) std::copy(all.begin(), all.end(), hits);
    return CMGPU_OK;
}

extern "C" int cmgpu_hb_stats(const cmgpu_model *m, double *kernel_ms, int64_t *cells, int32_t *launches) {
    if (!m) return CMGPU_EINVAL;
    const HbDev *h = m->hb;
    if (kernel_ms) *kernel_ms = h ? h->last_ms : 0.0;
    if (cells) *cells = h ? h->last_cells : 0;
    if (launches) *launches = h ? h->last_launches : 0;
    return CMGPU_OK;
}

extern "C" int cmgpu_tr_scan_hb_batch(const cmgpu_model *m, void *stream, int semiring, const cmgpu_tr_tables *tt,
                                      int pass_idx, int do_null3, const uint8_t *dsq_all, int64_t dsq_len,
                                      const cmgpu_tr_task *tasks, int32_t ntask, cmgpu_tr_result *results,
                                      cmgpu_tr_hit *hits, int64_t cap, int64_t *n_out) {
    if (!m || !dsq_all || ntask < 0 || (ntask > 0 && (!tasks || !results)) || !n_out) return CMGPU_EINVAL;
    *n_out = 0;
    if (ntask == 0) return CMGPU_OK;
    std::vector<cmgpu_tr_hit> all;
    int rc = tr_batch(m, (cudaStream_t)stream, semiring, tt, pass_idx, 1, do_null3, dsq_all, dsq_len, tasks, ntask,
                      results, all);
    if (rc) return rc;
    *n_out = (int64_t)all.size();
    if ((int64_t)all.size() > cap) {
        set_error("cmgpu_tr_scan_hb_batch: hit capacity too small");
        return CMGPU_EOVERFLOW;
    }
    if (hits) std::copy(all.begin(), all.end(), hits);
    return CMGPU_OK;
}

extern "C" int cmgpu_tr_scan_hb(const cmgpu_model *m, int semiring, const cmgpu_tr_tables *tt,
                                const cmgpu_hb_bands *bands, const uint8_t *jvalid, const uint8_t *lvalid,
                                const uint8_t *rvalid, const uint8_t *tvalid, const uint8_t *dsq, int32_t n,
                                int32_t i0, int32_t j0, float cutoff, int do_null3, int pass_idx, float env_cutoff,
                                float *vsc_root, int32_t *vmode, int64_t *envi, int64_t *envj, cmgpu_tr_hit *hits,
                                int32_t cap, int32_t *n_out) {
    if (!m || !bands || !dsq || n < 0 || !vsc_root || !vmode || !envi || !envj || !n_out) return CMGPU_EINVAL;
    *n_out = 0;
    cmgpu_tr_task tk{0, i0, j0, env_cutoff, cutoff, *bands, jvalid, lvalid, rvalid, tvalid};
    cmgpu_tr_result r{};
    std::vector<cmgpu_tr_hit> all;
    int rc = tr_batch(m, nullptr, semiring, tt, pass_idx, 1, do_null3, dsq, (int64_t)n + 2, &tk, 1, &r, all);
    if (rc) return rc;
    *vsc_root = r.vsc_root;
    *vmode = r.vmode;
    *envi = r.envi;
    *envj = r.envj;
    *n_out = (int32_t)all.size();
    if ((int64_t)all.size() > cap) {
        set_error("cmgpu_tr_scan_hb: hit capacity too small");
        return CMGPU_EOVERFLOW;
    }
    if (hits) std::copy(all.begin(), all.end(), hits);
    return CMGPU_OK;
}
