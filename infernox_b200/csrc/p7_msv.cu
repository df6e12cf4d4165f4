// P7 MSV / SSV filter (F1): 8-bit saturating MSV score of whole windows, and
// the SSV longtarget diagonal scan that turns chunks into candidate windows.
//
// Host side: the filter tables are built as the reference builds them
// (build_msv_filter, src/cm_pipeline.rs:201-340): emission scores byteified
// at 3/ln 2 with the bias from the best match score, the B->M, E->C and J->B
// move costs, and the prefix/suffix window-extension lengths; the windows
// found on the device are extended, merged and split on the host
// (extend_and_merge :722, split_windows :817).
//
// Device side.  A row i of the MSV/SSV matrix holds M cells; cell k reads
// only cell k-1 of row i-1 (plus the scalar B value), so a row is a shifted
// copy of the previous one.  One warp owns a row: lane l holds cells
// 1+2Rl .. 2R(l+1) in R registers, two 16-bit cells per register (values
// stay in 0..510, so 16-bit lanes never overflow), and the shift across a
// register pair is one byte permute; the cell k-1 of the first register
// comes from the neighbouring lane by one shuffle.  The u8 saturating ops of
// the reference -- max(dp, xB), +bias saturating at 255, -cost floored at
// 0 -- are packed s16x2 max/add/min/max.relu.
//
//  * MSV score: one warp per window, rows in order; xE is a warp max per row
//    because xJ and xB feed the next row.
//  * SSV scan: xB is constant, so a row depends only on the M-1 rows before
//    it.  A chunk is cut into segments, each scanned by one warp from zero
//    M-1 rows before its first row: the segment's rows then equal the rows of
//    a scan that never resets.  Every row whose xE reaches the trigger
//    threshold becomes a candidate (row, xE, leftmost argmax).  A reset only
//    lowers later rows (the recurrence is monotone and the reset state is the
//    floor), so the reference's triggers are a subset of the candidates.
//  * SSV replay: one warp per chunk walks the candidates in row order with
//    the reference's sequential logic: a candidate at least M-1 rows past the
//    last reset (or before any reset) is a trigger as it stands; nearer ones
//    are recomputed from the reset; a trigger is traced back and extended by
//    lane 0 (the reference's diagonal recovery) and the scan skips past it.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "../../include/cmscan_gpu.h"
#include "devbuf.h"

namespace cmx {
void set_error(const std::string &msg);
}

namespace {

constexpr int KP = 18;

// unbiased_byteify (src/cm_pipeline.rs:146-150)
uint8_t unbiased_byteify(float scale_b, float sc) {
    const float v = -roundf(scale_b * sc);
    if (v >= 255.0f) return 255;
    if (v <= 0.0f) return 0;
    return (uint8_t)v;
}

// biased_byteify (src/cm_pipeline.rs:164-172)
uint8_t biased_byteify(float scale_b, uint8_t bias_b, float sc) {
    const float v = -roundf(scale_b * sc);
    if (v > (float)(255 - (int)bias_b)) return 255;
    return (uint8_t)std::min(255, std::max(0, (int)v + (int)bias_b));
}

// canonical residues of each RNA code (src/cm_pipeline.rs:128-144)
const int DEGEN[KP][5] = {
    {1, 0}, {1, 1}, {1, 2}, {1, 3}, {0},      {2, 0, 2}, {2, 1, 3}, {2, 0, 1}, {2, 2, 3},
    {2, 1, 2}, {2, 0, 3}, {3, 0, 1, 3}, {3, 1, 2, 3}, {3, 0, 1, 2}, {3, 0, 2, 3}, {4, 0, 1, 2, 3}, {0}, {0}};

struct MsvHost {
    int M = 0, max_length = 0;
    float scale_b = 0;
    uint8_t base_b = 190, bias_b = 0, tbm_b = 0, tec_b = 0, tjb_b = 0;
    std::vector<uint8_t> rbv;           // [(M+1) * 18] emission costs
    std::vector<float> prefix, suffix;  // [M+1]
    double mmu = 0, mlambda = 1;
};

bool build_msv(const cmgpu_p7_profile *p, int max_length, double mmu, double mlambda, MsvHost &f) {
    const int m = p->M;
    if (m < 1 || !p->mat || !p->trans || max_length < 0) return false;
    f.M = m;
    f.max_length = max_length;
    f.mmu = mmu;
    f.mlambda = mlambda;
    f.scale_b = (float)(3.0 / 0.6931471805599453);
    f.base_b = 190;
    std::vector<float> msc((size_t)(m + 1) * KP, -INFINITY);
    float maxsc = 0.0f;
    for (int k = 1; k <= m; k++) {
        float *sc = &msc[(size_t)k * KP];
        for (int x = 0; x < 4; x++) {
            sc[x] = (float)std::log((double)p->mat[k * 4 + x] / 0.25);
            maxsc = std::max(maxsc, sc[x]);
        }
        for (int code = 4; code < KP; code++) {
            const int n = DEGEN[code][0];
            if (n == 0) continue;
            float s = 0.0f;
            for (int q = 0; q < n; q++) s += sc[DEGEN[code][1 + q]];
            sc[code] = s / (float)n;
        }
    }
    f.bias_b = unbiased_byteify(f.scale_b, -maxsc);
    f.rbv.assign((size_t)(m + 1) * KP, 255);
    for (int k = 1; k <= m; k++)
        for (int x = 0; x < KP; x++) f.rbv[(size_t)k * KP + x] = biased_byteify(f.scale_b, f.bias_b, msc[(size_t)k * KP + x]);
    f.tbm_b = unbiased_byteify(f.scale_b, (float)std::log(2.0 / ((double)m * ((double)m + 1.0))));
    f.tec_b = unbiased_byteify(f.scale_b, logf(0.5f));
    f.tjb_b = unbiased_byteify(f.scale_b, (float)std::log(3.0 / ((double)max_length + 3.0)));
    // window-extension lengths (src/cm_pipeline.rs:292-325)
    f.prefix.assign(m + 1, 0.0f);
    f.suffix.assign(m + 1, 0.0f);
    auto tr = [&](int k, int t) { return (double)p->trans[k * 7 + t]; };
    float sum = 0.0f;
    for (int k = 1; k < m; k++) {
        float v = 1.0f;
        if (tr(k, 1) != 0.0) {
            const double lii = std::log(tr(k, 4));
            if (lii != 0.0 && std::isfinite(lii)) v = (float)(1.0 + std::trunc(std::log(1e-7 / tr(k, 1)) / lii));
        }
        f.prefix[k] = v;
        sum += v;
    }
    if (sum > 0.0f)
        for (int k = 1; k < m; k++) f.prefix[k] /= sum;
    f.suffix[m] = f.prefix[m - 1];
    for (int k = m - 1; k >= 1; k--) f.suffix[k] = f.suffix[k + 1] + f.prefix[k - 1];
    for (int k = 2; k < m; k++) f.prefix[k] += f.prefix[k - 1];
    return true;
}

// the trigger threshold of ssv_diagonals (src/cm_pipeline.rs:522-533), with
// esl_gumbel_invsurv (src/easel/gumbel.rs:168-179)
int ssv_threshold(const MsvHost &f, double f1) {
    const double p1 = (double)f.max_length / ((double)f.max_length + 1.0);
    const double nullsc = (double)f.max_length * std::log(p1) + std::log(1.0 - p1);
    const double lp = f1 < 5e-9 ? (std::pow(f1, f1) - 1.0) / f1 : std::log(-std::log(1.0 - f1));
    const double invp = f.mmu - lp / f.mlambda;
    return (int)std::ceil((nullsc + invp * 0.6931471805599453 + 3.0) * (double)f.scale_b + (double)f.base_b +
                          (double)f.tec_b + (double)f.tjb_b);
}

// words (two cells each) per lane for a model of M positions
int words_for(int M) {
    static const int RS[] = {1, 2, 3, 4, 6, 8, 12, 16, 24, 32};
    const int need = (M + 63) / 64;
    for (int r : RS)
        if (r >= need) return r;
    return 0;
}

}  // namespace

struct cmgpu_msv_filter {
    int device = 0;
    int R = 0;
    MsvHost host;
    uint32_t *d_negc = nullptr;  // [18][R][32] packed s16x2 of -cost
    uint8_t *d_rbv = nullptr;    // [(M+1) * 18]
    mutable double last_ms = 0;
    mutable int64_t last_cells = 0;
    mutable int32_t last_launches = 0;
    mutable cmx::DevArena arena;  // per-call buffers, reused
    mutable cmx::PinnedBuf raw_pin;  // per-call host copy of the chunks' windows
    mutable int cap_hint = 64;    // candidate slots per segment the last scan needed
    ~cmgpu_msv_filter() {
        arena.release();
        cudaFree(d_negc);
        cudaFree(d_rbv);
    }
};

namespace cmx {
namespace dev {

constexpr unsigned FULL = 0xffffffffu;

__device__ __forceinline__ uint32_t add2(uint32_t a, uint32_t b) {
    uint32_t r;
    asm("add.s16x2 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
    return r;
}
__device__ __forceinline__ uint32_t max2(uint32_t a, uint32_t b) {
    uint32_t r;
    asm("max.s16x2 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
    return r;
}
__device__ __forceinline__ uint32_t min2(uint32_t a, uint32_t b) {
    uint32_t r;
    asm("min.s16x2 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
    return r;
}
__device__ __forceinline__ uint32_t relu2(uint32_t a) {
    uint32_t r;
    asm("max.relu.s16x2 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(0u));
    return r;
}
__device__ __forceinline__ uint32_t pack2(int v) { return ((uint32_t)v << 16) | (uint32_t)v; }

// One row of the shifted recurrence for lane `lane`:
//   w'[k] = max(min(max(w[k-1] + bias, xB + bias), 255) - cost[k][x], 0)
// negc points at this residue's packed -cost words, [r * 32 + lane].
// Returns the lane's packed maximum.
template <int R>
__device__ __forceinline__ uint32_t msv_row(uint32_t (&w)[R], const uint32_t *negc, int lane, uint32_t bias2,
                                            uint32_t xbb2) {
    uint32_t carry = __shfl_up_sync(FULL, w[R - 1], 1);
    if (lane == 0) carry = 0;
    const uint32_t c255 = 0x00ff00ffu;
    uint32_t mx = 0;
#pragma unroll
    for (int r = R - 1; r >= 0; r--) {
        const uint32_t prev = __byte_perm(r ? w[r - 1] : carry, w[r], 0x5432);
        uint32_t t = min2(max2(add2(prev, bias2), xbb2), c255);
        t = relu2(add2(t, negc[r * 32 + lane]));
        w[r] = t;
        mx = max2(mx, t);
    }
    return mx;
}

__device__ __forceinline__ int half_max(uint32_t v) { return max((int)(v & 0xffffu), (int)(v >> 16)); }

__device__ __forceinline__ int warp_max(int v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(FULL, v, o));
    return v;
}
__device__ __forceinline__ int warp_min(int v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = min(v, __shfl_xor_sync(FULL, v, o));
    return v;
}

// leftmost model position k (1-based) whose cell equals xe, over the warp
template <int R>
__device__ __forceinline__ int leftmost_k(const uint32_t (&w)[R], int lane, int xe) {
    int kk = INT_MAX;
#pragma unroll
    for (int r = R - 1; r >= 0; r--) {
        const int k0 = 1 + 2 * (lane * R + r);
        if ((int)(w[r] >> 16) == xe) kk = k0 + 1;
        if ((int)(w[r] & 0xffffu) == xe) kk = k0;
    }
    return warp_min(kk);
}

__device__ __forceinline__ int warp_incl_sum(int v, int lane) {
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(FULL, v, o);
        if (lane >= o) v += t;
    }
    return v;
}
__device__ __forceinline__ int warp_incl_max(int v, int lane) {
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(FULL, v, o);
        if (lane >= o) v = max(v, t);
    }
    return v;
}
// emission cost of residue code `code` at model position k (255 for codes
// past the alphabet, as the reference's sentinel rule)
__device__ __forceinline__ int cost_of(const uint8_t *rbv_s, int k, int code) {
    return code < KP ? rbv_s[k * KP + code] : 255;
}

struct MsvWin {
    int64_t off;  // buffer index of local residue 1 minus 1
    int32_t l;
    int32_t tjb;  // J->B cost of this window's length model
};

// MSV score (msv_score_tjb, src/cm_pipeline.rs:412-452); out[w] = xJ, or -1
// on overflow.
template <int R>
__global__ void __launch_bounds__(256) msv_score_kernel(const uint32_t *__restrict__ negc_g, int bias, int tec,
                                                        int base, int tbm, const uint8_t *__restrict__ dsq,
                                                        const MsvWin *__restrict__ wins, int nwin, int *out) {
    extern __shared__ uint32_t negc[];
    for (int q = threadIdx.x; q < KP * R * 32; q += blockDim.x) negc[q] = negc_g[q];
    __syncthreads();
    const int lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    const uint32_t bias2 = pack2(bias);
    for (int wi = blockIdx.x * nw + (threadIdx.x >> 5); wi < nwin; wi += gridDim.x * nw) {
        const MsvWin win = wins[wi];
        const uint8_t *frame = dsq + win.off;
        const int tjbm = (win.tjb + tbm) & 255;  // u8 wrapping sum
        uint32_t w[R];
#pragma unroll
        for (int r = 0; r < R; r++) w[r] = 0;
        int xj = 0, xb = max(base - tjbm, 0);
        bool overflow = false;
        uint32_t xs = 0;
        for (int i = 1; i <= win.l; i++) {
            const int q = (i - 1) & 31;
            if (q == 0) xs = (i + lane <= win.l) ? frame[i + lane] : 0;
            const int x = __shfl_sync(FULL, (int)xs, q);
            const uint32_t mx = msv_row<R>(w, negc + x * R * 32, lane, bias2, pack2(xb + bias));
            int xe = warp_max(half_max(mx));
            if (xe + bias >= 255) {
                overflow = true;
                break;
            }
            xe = max(xe - tec, 0);
            xj = max(xj, xe);
            xb = max(max(base, xj) - tjbm, 0);
        }
        if (lane == 0) out[wi] = overflow ? -1 : xj;
    }
}

struct SsvSeg {
    int64_t off;  // buffer index of local residue 1 minus 1
    int32_t r0, r1, w0, pad;
};

struct SsvCand {
    int32_t row;
    int16_t xe, k;
};

struct SsvChunk {
    int64_t off;
    int32_t l, seg_first, seg_count, pad;
};

struct SsvRaw {
    int32_t n, length, k;
    float score;
};

// Free-running SSV rows of one segment per warp; candidate rows (xE >=
// thr, thr >= 1) go to cands[seg * cap ...], their count to counts[seg].
template <int R>
__global__ void __launch_bounds__(256) ssv_scan_kernel(const uint32_t *__restrict__ negc_g, int bias, int xbb,
                                                       int thr, const uint8_t *__restrict__ dsq,
                                                       const SsvSeg *__restrict__ segs, int nseg, int cap,
                                                       SsvCand *cands, int *counts) {
    extern __shared__ uint32_t negc[];
    for (int q = threadIdx.x; q < KP * R * 32; q += blockDim.x) negc[q] = negc_g[q];
    __syncthreads();
    const int lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    const uint32_t bias2 = pack2(bias), xbb2 = pack2(xbb);
    for (int s = blockIdx.x * nw + (threadIdx.x >> 5); s < nseg; s += gridDim.x * nw) {
        const SsvSeg sg = segs[s];
        const uint8_t *frame = dsq + sg.off;
        uint32_t w[R];
#pragma unroll
        for (int r = 0; r < R; r++) w[r] = 0;
        int cnt = 0;
        uint32_t xs = 0;
        for (int i = sg.w0; i <= sg.r1; i++) {
            const int q = (i - sg.w0) & 31;
            if (q == 0) xs = (i + lane <= sg.r1) ? frame[i + lane] : 0;
            const int x = __shfl_sync(FULL, (int)xs, q);
            const uint32_t mx = msv_row<R>(w, negc + x * R * 32, lane, bias2, xbb2);
            const int lm = half_max(mx);
            if (__any_sync(FULL, lm >= thr) && i >= sg.r0) {
                const int xe = warp_max(lm);
                const int k = leftmost_k<R>(w, lane, xe);
                if (lane == 0 && cnt < cap) cands[(int64_t)s * cap + cnt] = SsvCand{i, (int16_t)xe, (int16_t)k};
                cnt++;
            }
        }
        if (lane == 0) counts[s] = cnt;
    }
}

// Sequential trigger logic of ssv_diagonals over one chunk per warp.
template <int R>
__global__ void __launch_bounds__(128) ssv_replay_kernel(const uint32_t *__restrict__ negc, const uint8_t *__restrict__ rbv,
                                                         int M, int bias, int xbb, int thr, int base, int tjb,
                                                         int tbm, float scale_b, const uint8_t *__restrict__ dsq,
                                                         const SsvChunk *__restrict__ chunks, int nchunk, int cap,
                                                         const SsvCand *__restrict__ cands,
                                                         const int *__restrict__ counts, SsvRaw *raws, int *nraw,
                                                         int *need) {
    extern __shared__ uint8_t rbv_s[];  // emission costs [(M+1) * 18]
    for (int q = threadIdx.x; q < (M + 1) * KP; q += blockDim.x) rbv_s[q] = rbv[q];
    __syncthreads();
    const int lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    const uint32_t bias2 = pack2(bias), xbb2 = pack2(xbb);
    for (int c = blockIdx.x * nw + (threadIdx.x >> 5); c < nchunk; c += gridDim.x * nw) {
        const SsvChunk ch = chunks[c];
        const uint8_t *frame = dsq + ch.off;
        bool bad = false;
        for (int s = ch.seg_first; s < ch.seg_first + ch.seg_count; s++)
            if (counts[s] > cap) {
                bad = true;
                if (lane == 0) atomicMax(need, counts[s]);
            }
        if (bad) {
            if (lane == 0) nraw[c] = 0;
            continue;
        }
        uint32_t w[R];
        int z = 1, i = 1, hz = -1, hr = 0, nr = 0;
        SsvRaw *out = raws + (int64_t)ch.seg_first * cap;
        for (int s = ch.seg_first; s < ch.seg_first + ch.seg_count; s++) {
            const int cnt = counts[s];
            for (int ci = 0; ci < cnt; ci++) {
                const SsvCand cd = cands[(int64_t)s * cap + ci];
                const int r = cd.row;
                if (r < i) continue;
                int xe = cd.xe, ek = cd.k;
                if (z != 1 && r < z + M - 1) {
                    // rows since the reset at z differ from the free-running
                    // ones: recompute them from the zero state
                    if (hz != z) {
#pragma unroll
                        for (int q = 0; q < R; q++) w[q] = 0;
                        hz = z;
                        hr = z - 1;
                    }
                    uint32_t mx = 0;
                    for (int rr = hr + 1; rr <= r; rr++) mx = msv_row<R>(w, negc + frame[rr] * R * 32, lane, bias2, xbb2);
                    hr = r;
                    xe = warp_max(half_max(mx));
                    if (xe < thr) continue;
                    ek = leftmost_k<R>(w, lane, xe);
                }
                // trigger at row r: recover the diagonal and extend it
                // (src/cm_pipeline.rs:637-705), 32 steps at a time
                int start, tstart, max_sc = xe, max_end = r;
                {
                    // backward: step s reads (ek - s, r - s) while rem > baseline
                    const int baseline = base - tjb - tbm;
                    int taken = 0, rem = xe;
                    for (;;) {
                        const int kk = ek - taken - lane, tt = r - taken - lane;
                        const bool valid = kk >= 1 && tt >= 1;
                        const int delta = valid ? bias - cost_of(rbv_s, kk, frame[tt]) : 0;
                        const int incl = warp_incl_sum(delta, lane);
                        const bool cont = valid && rem - (incl - delta) > baseline;
                        const unsigned stop = __ballot_sync(FULL, !cont);
                        if (stop) {
                            taken += __ffs(stop) - 1;
                            break;
                        }
                        taken += 32;
                        rem -= __shfl_sync(FULL, incl, 31);
                    }
                    start = ek - taken + 1;
                    tstart = r - taken + 1;
                    // forward: running score, new maxima reset the miss count,
                    // the fifth miss in a row (or the model / chunk end) stops
                    int t0 = 0, base_sc = xe, runmax = xe, since = 0;
                    for (;;) {
                        const int k = ek + 1 + t0 + lane, n = r + 1 + t0 + lane;
                        const bool valid = k < M && n <= ch.l;
                        const int delta = valid ? bias - cost_of(rbv_s, k, frame[n]) : 0;
                        const int sc = base_sc + warp_incl_sum(delta, lane);
                        int pm = warp_incl_max(sc, lane);
                        int before = __shfl_up_sync(FULL, pm, 1);
                        before = lane == 0 ? runmax : max(runmax, before);
                        const bool imp = valid && sc >= before;
                        const unsigned impm = __ballot_sync(FULL, imp);
                        const unsigned upto = lane == 31 ? 0xffffffffu : ((1u << (lane + 1)) - 1u);
                        const unsigned mine = impm & upto;
                        const int since_t = mine ? lane - (31 - __clz(mine)) : since + lane + 1;
                        const bool halt = !valid || (!imp && since_t == 5);
                        const unsigned hm = __ballot_sync(FULL, halt);
                        const int q = hm ? __ffs(hm) - 1 : 32;          // first lane that ends the walk
                        const unsigned before_q = q == 32 ? impm : (impm & ((1u << q) - 1u));
                        if (before_q) {
                            const int pl = 31 - __clz(before_q);      // last new maximum before the end
                            max_sc = __shfl_sync(FULL, sc, pl);
                            max_end = r + 1 + t0 + pl;
                        }
                        if (hm) break;
                        since = impm ? 31 - (31 - __clz(impm)) : since + 32;
                        runmax = max(runmax, __shfl_sync(FULL, pm, 31));
                        base_sc = __shfl_sync(FULL, sc, 31);
                        t0 += 32;
                    }
                }
                if (lane == 0) {
                    const int end_model = ek + (max_end - r);
                    const float sc = (__fsub_rn((float)(max_sc - tjb), (float)base) / scale_b) - 3.0f;
                    out[nr] = SsvRaw{tstart, end_model - start + 1, end_model, sc};
                }
                nr++;
                z = max_end + 1;
                i = max_end + 1;
            }
        }
        if (lane == 0) nraw[c] = nr;
    }
}

}  // namespace dev
}  // namespace cmx

using namespace cmx;

namespace {

#define MSV_TRY(call)                                                                           \
    do {                                                                                        \
        cudaError_t e_ = (call);                                                                \
        if (e_ != cudaSuccess) {                                                                \
            set_error(std::string("msv: ") + #call + ": " + cudaGetErrorString(e_));            \
            return CMGPU_EDEVICE;                                                               \
        }                                                                                       \
    } while (0)

#define MSV_ALLOC(slot, ptr, bytes)                                                             \
    do {                                                                                        \
        cudaError_t e_ = f->arena.get((slot), &(ptr), (bytes));                                 \
        if (e_ != cudaSuccess) {                                                                \
            set_error(std::string("msv: device allocation: ") + cudaGetErrorString(e_));        \
            return CMGPU_ENOMEM;                                                                \
        }                                                                                       \
    } while (0)

int check_windows(const char *who, const uint8_t *dsq_all, int64_t dsq_len, const cmgpu_window *wins, int32_t n) {
    for (int32_t k = 0; k < n; k++) {
        const cmgpu_window &w = wins[k];
        if (w.dsq_offset < 0 || w.i0 < 1 || w.j0 < w.i0 - 1 || w.dsq_offset + (int64_t)w.j0 + 1 > dsq_len) {
            set_error(std::string(who) + ": window outside the residue buffer");
            return CMGPU_EINVAL;
        }
        if (w.j0 >= w.i0 && any_code_above_17(dsq_all + w.dsq_offset + w.i0, (int64_t)w.j0 - w.i0 + 1)) {
            set_error(std::string(who) + ": residue code > 17");
            return CMGPU_EINVAL;
        }
    }
    return CMGPU_OK;
}

template <int R>
void launch_msv(const cmgpu_msv_filter *f, cudaStream_t st, const uint8_t *d_dsq, const dev::MsvWin *d_w, int n,
                int *d_out, int grid) {
    const size_t smem = (size_t)KP * R * 32 * sizeof(uint32_t);
    cmx::allow_max_dynamic_smem(dev::msv_score_kernel<R>);
    const MsvHost &h = f->host;
    dev::msv_score_kernel<R><<<grid, 256, smem, st>>>(f->d_negc, h.bias_b, h.tec_b, h.base_b, h.tbm_b, d_dsq, d_w, n,
                                                      d_out);
}

template <int R>
void launch_ssv(const cmgpu_msv_filter *f, cudaStream_t st, int xbb, int thr, const uint8_t *d_dsq,
                const dev::SsvSeg *d_segs, int nseg, const dev::SsvChunk *d_ch, int nch, int cap,
                dev::SsvCand *d_cands, int *d_counts, dev::SsvRaw *d_raws, int *d_nraw, int *d_need) {
    const size_t smem = (size_t)KP * R * 32 * sizeof(uint32_t);
    cmx::allow_max_dynamic_smem(dev::ssv_scan_kernel<R>);
    const MsvHost &h = f->host;
    dev::ssv_scan_kernel<R><<<(nseg + 7) / 8, 256, smem, st>>>(f->d_negc, h.bias_b, xbb, thr, d_dsq, d_segs, nseg, cap,
                                                              d_cands, d_counts);
    const size_t rsm = (size_t)(h.M + 1) * KP;
    cmx::allow_max_dynamic_smem(dev::ssv_replay_kernel<R>);
    dev::ssv_replay_kernel<R><<<(nch + 3) / 4, 128, rsm, st>>>(f->d_negc, f->d_rbv, h.M, h.bias_b, xbb, thr, h.base_b,
                                                            h.tjb_b, h.tbm_b, h.scale_b, d_dsq, d_ch, nch, cap, d_cands,
                                                            d_counts, d_raws, d_nraw, d_need);
}

#define DISPATCH_R(R, CALL)                  \
    switch (R) {                             \
        case 1: CALL(1); break;              \
        case 2: CALL(2); break;              \
        case 3: CALL(3); break;              \
        case 4: CALL(4); break;              \
        case 6: CALL(6); break;              \
        case 8: CALL(8); break;              \
        case 12: CALL(12); break;            \
        case 16: CALL(16); break;            \
        case 24: CALL(24); break;            \
        default: CALL(32); break;            \
    }

struct RawWin {
    int64_t n, length, k;
    float score;
};

// extend_and_merge with pct_overlap 0 and split_windows (src/cm_pipeline.rs:722-840)
void extend_merge_split(const MsvHost &f, std::vector<RawWin> &raws, int64_t target_len, int64_t cmw, int32_t chunk,
                        std::vector<cmgpu_f1_window> &out) {
    if (raws.empty()) return;
    const double maxl = (double)f.max_length;
    for (RawWin &w : raws) {
        const int64_t ks = std::clamp<int64_t>(w.k - w.length + 1, 0, f.M), ke = std::clamp<int64_t>(w.k, 0, f.M);
        const double ws = std::max((double)w.n - maxl * (0.1 + (double)f.prefix[ks]), 1.0);
        const double we = std::min((double)w.n + (double)w.length + maxl * (0.1 + (double)f.suffix[ke]),
                                   (double)target_len);
        const int64_t s = (int64_t)ws, e = (int64_t)we;
        w.n = s;
        w.length = e - s + 1;
    }
    std::vector<RawWin> kept{raws[0]};
    for (size_t q = 1; q < raws.size(); q++) {
        const RawWin cur = raws[q];
        RawWin &prev = kept.back();
        const int64_t pe = prev.n + prev.length - 1, ce = cur.n + cur.length - 1;
        const int64_t wl = std::min(pe, ce) - std::max(prev.n, cur.n) + 1;
        const int64_t minlen = std::min(prev.length, cur.length);
        if ((float)wl / (float)minlen > 0.0f) {
            const int64_t ms = std::min(prev.n, cur.n);
            prev.length = std::max(pe, ce) - ms + 1;
            prev.n = ms;
        } else {
            kept.push_back(cur);
        }
    }
    for (const RawWin &w : kept) {
        const int64_t ws = w.n, we = w.n + w.length - 1;
        if (we - ws + 1 > 2 * cmw) {
            int64_t s = ws, e = std::min(ws + 2 * cmw - 1, we);
            out.push_back(cmgpu_f1_window{s, e, w.score, chunk});
            while (e < we) {
                s = std::min(s + cmw, we);
                e = std::min(e + cmw, we);
                out.push_back(cmgpu_f1_window{s, e, w.score, chunk});
            }
        } else {
            out.push_back(cmgpu_f1_window{ws, we, w.score, chunk});
        }
    }
}

// the device part shared by cmgpu_ssv_diagonals and cmgpu_f1_msv_windows:
// raw diagonals per chunk, in the order ssv_diagonals finds them
int ssv_run(const cmgpu_msv_filter *f, cudaStream_t st, const uint8_t *dsq_all, int64_t dsq_len,
            const cmgpu_window *chunks, int32_t nch, double f1, std::vector<std::vector<RawWin>> &raws) {
    const MsvHost &h = f->host;
    const int M = h.M;
    const int thr = std::max(ssv_threshold(h, f1), 1);
    const int xb = std::max((int)h.base_b - std::min((int)h.tjb_b + (int)h.tbm_b, 255), 0);
    const int xbb = xb + h.bias_b;
    raws.assign(nch, {});
    // segments: long enough to amortise the M-1 warm-up rows, short enough to
    // give every SM several warps
    int64_t total = 0;
    for (int32_t c = 0; c < nch; c++) total += std::max(0, chunks[c].j0 - chunks[c].i0 + 1);
    int64_t seg_len = std::clamp<int64_t>(total / (148 * 48) + 1, 256, 8192);
    seg_len = std::max<int64_t>(seg_len, 2 * (int64_t)M);
    std::vector<dev::SsvSeg> segs;
    std::vector<dev::SsvChunk> ch(nch);
    for (int32_t c = 0; c < nch; c++) {
        const int32_t l = std::max(0, chunks[c].j0 - chunks[c].i0 + 1);
        const int64_t off = chunks[c].dsq_offset + chunks[c].i0 - 1;
        ch[c] = dev::SsvChunk{off, l, (int32_t)segs.size(), 0, 0};
        for (int64_t r0 = 1; r0 <= l; r0 += seg_len) {
            const int32_t r1 = (int32_t)std::min<int64_t>(l, r0 + seg_len - 1);
            segs.push_back(dev::SsvSeg{off, (int32_t)r0, r1, (int32_t)std::max<int64_t>(1, r0 - (M - 1)), 0});
        }
        ch[c].seg_count = (int32_t)segs.size() - ch[c].seg_first;
    }
    const int nseg = (int)segs.size();
    if (nseg == 0) return CMGPU_OK;
    uint8_t *d_dsq;
    dev::SsvSeg *d_segs;
    dev::SsvChunk *d_ch;
    int *d_counts, *d_nraw, *d_need;
    MSV_ALLOC(0, d_dsq, (size_t)dsq_len);
    MSV_ALLOC(1, d_segs, sizeof(dev::SsvSeg) * nseg);
    MSV_ALLOC(2, d_ch, sizeof(dev::SsvChunk) * nch);
    MSV_ALLOC(3, d_counts, sizeof(int) * nseg);
    MSV_ALLOC(4, d_nraw, sizeof(int) * nch);
    MSV_ALLOC(5, d_need, sizeof(int));
    MSV_TRY(cudaMemcpyAsync(d_dsq, dsq_all, (size_t)dsq_len, cudaMemcpyHostToDevice, st));
    MSV_TRY(cudaMemcpyAsync(d_segs, segs.data(), sizeof(dev::SsvSeg) * nseg, cudaMemcpyHostToDevice, st));
    MSV_TRY(cudaMemcpyAsync(d_ch, ch.data(), sizeof(dev::SsvChunk) * nch, cudaMemcpyHostToDevice, st));
    cudaEvent_t e0, e1;
    MSV_TRY(cudaEventCreate(&e0));
    MSV_TRY(cudaEventCreate(&e1));
    int cap = f->cap_hint;
    double ms_total = 0;
    int launches = 0;
    for (int attempt = 0; attempt < 2; attempt++) {
        dev::SsvCand *d_cands;
        dev::SsvRaw *d_raws;
        cudaError_t e;
        if ((e = f->arena.get(6, &d_cands, sizeof(dev::SsvCand) * (size_t)nseg * cap)) != cudaSuccess ||
            (e = f->arena.get(7, &d_raws, sizeof(dev::SsvRaw) * (size_t)nseg * cap)) != cudaSuccess) {
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            set_error(std::string("msv: device allocation: ") + cudaGetErrorString(e));
            return CMGPU_ENOMEM;
        }
        MSV_TRY(cudaMemsetAsync(d_need, 0, sizeof(int), st));
        MSV_TRY(cudaEventRecord(e0, st));
#define CALL_SSV(RR) \
    launch_ssv<RR>(f, st, xbb, thr, d_dsq, d_segs, nseg, d_ch, nch, cap, d_cands, d_counts, d_raws, d_nraw, d_need)
        DISPATCH_R(f->R, CALL_SSV);
#undef CALL_SSV
        MSV_TRY(cudaGetLastError());
        MSV_TRY(cudaEventRecord(e1, st));
        int need = 0;
        std::vector<int> nraw(nch);
        MSV_TRY(cudaMemcpyAsync(&need, d_need, sizeof(int), cudaMemcpyDeviceToHost, st));
        MSV_TRY(cudaMemcpyAsync(nraw.data(), d_nraw, sizeof(int) * nch, cudaMemcpyDeviceToHost, st));
        MSV_TRY(cudaStreamSynchronize(st));
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        ms_total += ms;
        launches += 2;
        if (need > cap) {
            cap = need + need / 4;
            f->cap_hint = cap;
            continue;
        }
        // only each chunk's windows come back (they sit at the chunk's first
        // segment slot), into pinned memory
        size_t nall = 0;
        std::vector<size_t> at(nch);
        for (int32_t c = 0; c < nch; c++) {
            at[c] = nall;
            nall += (size_t)std::max(0, nraw[c]);
        }
        dev::SsvRaw *hr = f->raw_pin.get<dev::SsvRaw>(std::max<size_t>(nall, 1));
        if (!hr) {
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            set_error("msv: pinned host allocation failed");
            return CMGPU_ENOMEM;
        }
        for (int32_t c = 0; c < nch; c++)
            if (nraw[c] > 0)
                MSV_TRY(cudaMemcpyAsync(hr + at[c], d_raws + (size_t)ch[c].seg_first * cap,
                                        sizeof(dev::SsvRaw) * (size_t)nraw[c], cudaMemcpyDeviceToHost, st));
        MSV_TRY(cudaStreamSynchronize(st));
        for (int32_t c = 0; c < nch; c++) {
            const dev::SsvRaw *p = hr + at[c];
            for (int q = 0; q < nraw[c]; q++) raws[c].push_back(RawWin{p[q].n, p[q].length, p[q].k, p[q].score});
        }
        break;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    int64_t cells = 0;
    for (const dev::SsvSeg &s : segs) cells += (int64_t)(s.r1 - s.w0 + 1) * M;
    f->last_ms = ms_total;
    f->last_cells = cells;
    f->last_launches = launches;
    return CMGPU_OK;
}

}  // namespace

extern "C" int cmgpu_msv_filter_build(const cmgpu_p7_profile *p, int32_t max_length, double lmmu, double lmlambda,
                                      int device, cmgpu_msv_filter **out) {
    if (!p || !out) return CMGPU_EINVAL;
    *out = nullptr;
    std::unique_ptr<cmgpu_msv_filter> f(new cmgpu_msv_filter());
    f->device = device;
    if (!build_msv(p, max_length, lmmu, lmlambda, f->host)) {
        set_error("cmgpu_msv_filter_build: bad profile");
        return CMGPU_EINVAL;
    }
    f->R = words_for(p->M);
    if (f->R == 0) {
        set_error("cmgpu_msv_filter_build: models longer than 2048 positions are not supported");
        return CMGPU_ENOSPACE;
    }
    if (device >= 0) {  // device < 0: host tables only (no GPU needed)
        const int R = f->R, M = p->M;
        std::vector<uint32_t> negc((size_t)KP * R * 32);
        for (int x = 0; x < KP; x++)
            for (int r = 0; r < R; r++)
                for (int l = 0; l < 32; l++) {
                    const int k = 1 + 2 * (l * R + r);
                    const int c0 = k <= M ? f->host.rbv[(size_t)k * KP + x] : 255;
                    const int c1 = k + 1 <= M ? f->host.rbv[(size_t)(k + 1) * KP + x] : 255;
                    negc[((size_t)x * R + r) * 32 + l] = ((uint32_t)(uint16_t)(-c1) << 16) | (uint16_t)(-c0);
                }
        MSV_TRY(cudaSetDevice(device));
        MSV_TRY(cudaMalloc((void **)&f->d_negc, negc.size() * sizeof(uint32_t)));
        MSV_TRY(cudaMemcpy(f->d_negc, negc.data(), negc.size() * sizeof(uint32_t), cudaMemcpyHostToDevice));
        MSV_TRY(cudaMalloc((void **)&f->d_rbv, f->host.rbv.size()));
        MSV_TRY(cudaMemcpy(f->d_rbv, f->host.rbv.data(), f->host.rbv.size(), cudaMemcpyHostToDevice));
    }
    *out = f.release();
    return CMGPU_OK;
}

extern "C" void cmgpu_msv_filter_free(cmgpu_msv_filter *f) { delete f; }

extern "C" int cmgpu_msv_filter_tables(const cmgpu_msv_filter *f, uint8_t *rbv, int32_t cap, int32_t *n_out,
                                       uint8_t *bytes5, float *prefix, float *suffix, float *scale_b) {
    if (!f || !n_out) return CMGPU_EINVAL;
    const MsvHost &h = f->host;
    *n_out = (int32_t)h.rbv.size();
    if (bytes5) {
        bytes5[0] = h.base_b;
        bytes5[1] = h.bias_b;
        bytes5[2] = h.tbm_b;
        bytes5[3] = h.tec_b;
        bytes5[4] = h.tjb_b;
    }
    if (prefix) std::copy(h.prefix.begin(), h.prefix.end(), prefix);
    if (suffix) std::copy(h.suffix.begin(), h.suffix.end(), suffix);
    if (scale_b) *scale_b = h.scale_b;
    if ((int64_t)h.rbv.size() > cap) return CMGPU_EOVERFLOW;
    if (rbv) std::copy(h.rbv.begin(), h.rbv.end(), rbv);
    return CMGPU_OK;
}

extern "C" int cmgpu_ssv_threshold(const cmgpu_msv_filter *f, double f1, int32_t *thresh) {
    if (!f || !thresh) return CMGPU_EINVAL;
    *thresh = ssv_threshold(f->host, f1);
    return CMGPU_OK;
}

extern "C" int cmgpu_msv_filter_stats(const cmgpu_msv_filter *f, double *kernel_ms, int64_t *cells,
                                      int32_t *launches) {
    if (!f) return CMGPU_EINVAL;
    if (kernel_ms) *kernel_ms = f->last_ms;
    if (cells) *cells = f->last_cells;
    if (launches) *launches = f->last_launches;
    return CMGPU_OK;
}

extern "C" int cmgpu_msv_score_batch(const cmgpu_msv_filter *f, void *stream_ptr, const uint8_t *dsq_all,
                                     int64_t dsq_len, const cmgpu_window *wins, int32_t nwin, const int32_t *wlen,
                                     float *scores, uint8_t *scored) {
    if (!f || !dsq_all || nwin < 0 || (nwin > 0 && (!wins || !scores || !scored))) return CMGPU_EINVAL;
    if (!f->d_negc) {
        set_error("cmgpu_msv_score_batch: filter was built without a device");
        return CMGPU_EINVAL;
    }
    if (nwin == 0) return CMGPU_OK;
    int rc = check_windows("cmgpu_msv_score_batch", dsq_all, dsq_len, wins, nwin);
    if (rc) return rc;
    const MsvHost &h = f->host;
    std::vector<dev::MsvWin> vw(nwin);
    int64_t cells = 0;
    for (int32_t k = 0; k < nwin; k++) {
        const int32_t l = std::max(0, wins[k].j0 - wins[k].i0 + 1);
        const uint8_t tjb = wlen ? unbiased_byteify(h.scale_b, (float)std::log(3.0 / ((double)wlen[k] + 3.0))) : h.tjb_b;
        vw[k] = dev::MsvWin{wins[k].dsq_offset + wins[k].i0 - 1, l, tjb};
        cells += (int64_t)l * h.M;
    }
    cudaStream_t st = (cudaStream_t)stream_ptr;
    MSV_TRY(cudaSetDevice(f->device));
    uint8_t *d_dsq;
    dev::MsvWin *d_w;
    int *d_out;
    MSV_ALLOC(0, d_dsq, (size_t)dsq_len);
    MSV_ALLOC(8, d_w, sizeof(dev::MsvWin) * nwin);
    MSV_ALLOC(9, d_out, sizeof(int) * nwin);
    MSV_TRY(cudaMemcpyAsync(d_dsq, dsq_all, (size_t)dsq_len, cudaMemcpyHostToDevice, st));
    MSV_TRY(cudaMemcpyAsync(d_w, vw.data(), sizeof(dev::MsvWin) * nwin, cudaMemcpyHostToDevice, st));
    cudaEvent_t e0, e1;
    MSV_TRY(cudaEventCreate(&e0));
    MSV_TRY(cudaEventCreate(&e1));
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, f->device);
    const int grid = (int)std::min<int64_t>((nwin + 7) / 8, (int64_t)sms * 8);
    cudaEventRecord(e0, st);
#define CALL_MSV(RR) launch_msv<RR>(f, st, d_dsq, d_w, nwin, d_out, grid)
    DISPATCH_R(f->R, CALL_MSV);
#undef CALL_MSV
    cudaError_t e = cudaGetLastError();
    cudaEventRecord(e1, st);
    std::vector<int> out(nwin);
    if (e == cudaSuccess) e = cudaMemcpyAsync(out.data(), d_out, sizeof(int) * nwin, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    float ms = 0;
    if (e == cudaSuccess) cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (e != cudaSuccess) {
        set_error(std::string("cmgpu_msv_score_batch: ") + cudaGetErrorString(e));
        return CMGPU_EDEVICE;
    }
    f->last_ms = ms;
    f->last_cells = cells;
    f->last_launches = 1;
    // ret = ((xJ - tjb) - base) / scale_b - 3 (src/cm_pipeline.rs:450), in f32
    for (int32_t k = 0; k < nwin; k++) {
        scored[k] = out[k] >= 0;
        scores[k] = out[k] >= 0 ? ((float)(out[k] - vw[k].tjb) - (float)h.base_b) / h.scale_b - 3.0f : NAN;
    }
    return CMGPU_OK;
}

extern "C" int cmgpu_ssv_diagonals(const cmgpu_msv_filter *f, void *stream, const uint8_t *dsq_all, int64_t dsq_len,
                                   const cmgpu_window *chunks, int32_t nchunk, double f1, cmgpu_ssv_diagonal *out,
                                   int32_t cap, int32_t *n_out) {
    if (!f || !dsq_all || nchunk < 0 || !n_out || (nchunk > 0 && !chunks)) return CMGPU_EINVAL;
    *n_out = 0;
    if (!f->d_negc) {
        set_error("cmgpu_ssv_diagonals: filter was built without a device");
        return CMGPU_EINVAL;
    }
    int rc = check_windows("cmgpu_ssv_diagonals", dsq_all, dsq_len, chunks, nchunk);
    if (rc) return rc;
    MSV_TRY(cudaSetDevice(f->device));
    std::vector<std::vector<RawWin>> raws;
    rc = ssv_run(f, (cudaStream_t)stream, dsq_all, dsq_len, chunks, nchunk, f1, raws);
    if (rc) return rc;
    int64_t n = 0;
    for (int32_t c = 0; c < nchunk; c++)
        for (const RawWin &w : raws[c]) {
            if (out && n < cap) out[n] = cmgpu_ssv_diagonal{w.n, w.length, w.k, w.score, c};
            n++;
        }
    *n_out = (int32_t)n;
    return n > cap ? CMGPU_EOVERFLOW : CMGPU_OK;
}

namespace cmx {
// f1_msv_windows on every chunk into a vector (windows grouped by chunk);
// the chunks have been checked by the caller.
int f1_msv_windows_vec(const cmgpu_msv_filter *f, cudaStream_t st, const uint8_t *dsq_all, int64_t dsq_len,
                       const cmgpu_window *chunks, int32_t nchunk, double f1, int64_t cmw,
                       std::vector<cmgpu_f1_window> &wins) {
    MSV_TRY(cudaSetDevice(f->device));
    std::vector<std::vector<RawWin>> raws;
    int rc = ssv_run(f, st, dsq_all, dsq_len, chunks, nchunk, f1, raws);
    if (rc) return rc;
    wins.clear();
    for (int32_t c = 0; c < nchunk; c++)
        extend_merge_split(f->host, raws[c], std::max(0, chunks[c].j0 - chunks[c].i0 + 1), cmw, c, wins);
    return CMGPU_OK;
}
}  // namespace cmx

extern "C" int cmgpu_f1_msv_windows(const cmgpu_msv_filter *f, void *stream, const uint8_t *dsq_all, int64_t dsq_len,
                                    const cmgpu_window *chunks, int32_t nchunk, double f1, int64_t cmw,
                                    cmgpu_f1_window *out, int32_t cap, int32_t *n_out) {
    if (!f || !dsq_all || nchunk < 0 || !n_out || (nchunk > 0 && !chunks) || cmw < 1) return CMGPU_EINVAL;
    *n_out = 0;
    if (!f->d_negc) {
        set_error("cmgpu_f1_msv_windows: filter was built without a device");
        return CMGPU_EINVAL;
    }
    int rc = check_windows("cmgpu_f1_msv_windows", dsq_all, dsq_len, chunks, nchunk);
    if (rc) return rc;
    std::vector<cmgpu_f1_window> wins;
    rc = cmx::f1_msv_windows_vec(f, (cudaStream_t)stream, dsq_all, dsq_len, chunks, nchunk, f1, cmw, wins);
    if (rc) return rc;
    *n_out = (int32_t)wins.size();
    if ((int64_t)wins.size() > cap) {
        set_error("cmgpu_f1_msv_windows: output capacity too small");
        return CMGPU_EOVERFLOW;
    }
    if (out) std::copy(wins.begin(), wins.end(), out);
    return CMGPU_OK;
}
