// P7 Viterbi filter (F2): int16 saturating local Viterbi score of whole
// windows, many windows per launch.
//
// Host side: the filter tables are built as the reference builds them
// (build_vit_filter, src/p7_vitfilter.rs:121-278): scores quantised by
// wordify (scale 500/ln2, round half away, saturate), into-M transitions
// capped at 0, II capped at -1, local entries from the match occupancy, and
// the per-length N/C/J move cost of vit_score_scalar (:305-385).
//
// Device side: one warp per window, rows i in order.  Model positions
// k = 1..M are split into blocks of consecutive positions, lane l owning
// block l.  For M <= 256 each lane keeps its block of the M, I and D rows in
// registers as packed pairs of int16 cells, and every saturating add and max
// acts on two cells at once (the sm_90+ add/max/min.s16x2 instructions, with
// the saturation done by clamping the operand first); longer models keep the
// rows in shared memory with a padded lane stride (conflict-free), one cell
// per 32-bit lane op.  M and I cells read only the previous row; xE is a warp
// max.  D cells form a serial chain along k in the same row (D(i,k) from
// M(i,k-1) and D(i,k-1)); each lane walks its block serially from an incoming
// value and the warp repeats until no incoming value changes -- the values
// then satisfy the serial chain, so they equal the scalar full DD sweep bit
// for bit (and the SSE lazy-F result, which the reference shows is the
// same).  All arithmetic is 16-bit saturating.
#include <cuda_runtime.h>

#include <algorithm>
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
constexpr int16_t NEGINF16 = -32768;

// wordify (src/p7_vitfilter.rs:55-68)
int16_t wordify(float scale_w, float sc) {
    if (sc == -INFINITY) return NEGINF16;
    float v = roundf(scale_w * sc);
    if (v >= 32767.0f) return 32767;
    if (v <= -32768.0f) return NEGINF16;
    return (int16_t)v;
}

// canonical residues of each RNA code (src/p7_vitfilter.rs:29-47)
const int DEGEN[KP][5] = {
    {1, 0}, {1, 1}, {1, 2}, {1, 3}, {0},      {2, 0, 2}, {2, 1, 3}, {2, 0, 1}, {2, 2, 3},
    {2, 1, 2}, {2, 0, 3}, {3, 0, 1, 3}, {3, 1, 2, 3}, {3, 0, 1, 2}, {3, 0, 2, 3}, {4, 0, 1, 2, 3}, {0}, {0}};

struct VitHost {
    int M = 0;
    float scale_w = 0;
    int16_t base_w = 0, e_move = 0, e_loop = 0;
    // per position k = 0..M: [0..17] emissions, then vbm, tmm, tim, tdm, tmi, tii, tmd, tdd
    std::vector<int16_t> tab;  // [(M+1) * 26]
};
constexpr int TAB_W = 26;
enum { T_VBM = 18, T_MM, T_IM, T_DM, T_MI, T_II, T_MD, T_DD };

bool build_vit(const cmgpu_p7_profile *p, VitHost &f) {
    const int m = p->M;
    if (m < 1 || !p->mat || !p->trans) return false;
    f.M = m;
    f.scale_w = (float)(500.0 / 0.6931471805599453);
    f.base_w = 12000;
    f.tab.assign((size_t)(m + 1) * TAB_W, NEGINF16);
    auto T = [&](int k, int c) -> int16_t & { return f.tab[(size_t)k * TAB_W + c]; };
    for (int k = 1; k <= m; k++) {
        float sc[KP];
        for (int x = 0; x < KP; x++) sc[x] = -INFINITY;
        for (int x = 0; x < 4; x++) sc[x] = (float)std::log((double)p->mat[k * 4 + x] / 0.25);
        for (int code = 4; code < KP; code++) {
            int n = DEGEN[code][0];
            if (n == 0) continue;
            float s = 0.0f;
            for (int q = 0; q < n; q++) s += sc[DEGEN[code][1 + q]];
            sc[code] = s / (float)n;
        }
        for (int x = 0; x < KP; x++) T(k, x) = wordify(f.scale_w, sc[x]);
    }
    auto tr = [&](int j, int t) { return p->trans[j * 7 + t]; };
    for (int j = 1; j < m; j++) {
        T(j, T_MM) = std::min<int16_t>(wordify(f.scale_w, (float)std::log((double)tr(j, 0))), 0);
        T(j, T_IM) = std::min<int16_t>(wordify(f.scale_w, (float)std::log((double)tr(j, 3))), 0);
        T(j, T_DM) = std::min<int16_t>(wordify(f.scale_w, (float)std::log((double)tr(j, 5))), 0);
        T(j, T_MI) = std::min<int16_t>(wordify(f.scale_w, (float)std::log((double)tr(j, 1))), 0);
        T(j, T_II) = std::min<int16_t>(wordify(f.scale_w, (float)std::log((double)tr(j, 4))), -1);
        T(j, T_MD) = std::min<int16_t>(wordify(f.scale_w, (float)std::log((double)tr(j, 2))), 0);
        T(j, T_DD) = std::min<int16_t>(wordify(f.scale_w, (float)std::log((double)tr(j, 6))), 0);
    }
    // local entry occupancy (src/p7_vitfilter.rs:186-201)
    std::vector<float> occ(m + 1, 0.0f);
    occ[1] = tr(0, 1) + tr(0, 0);
    for (int k = 2; k <= m; k++)
        occ[k] = occ[k - 1] * (tr(k - 1, 0) + tr(k - 1, 1)) + (1.0f - occ[k - 1]) * tr(k - 1, 5);
    float z = 0.0f;
    for (int k = 1; k <= m; k++) z += occ[k] * (float)(m - k + 1);
    for (int k = 1; k <= m; k++) {
        float logv = (float)std::log((double)(occ[k] / z));
        T(k, T_VBM) = std::min<int16_t>(wordify(f.scale_w, logv), 0);
    }
    f.e_move = wordify(f.scale_w, -(float)0.6931471805599453);
    f.e_loop = f.e_move;
    return true;
}

// per-length move cost (src/p7_vitfilter.rs:311-312)
int16_t xw_move_for(float scale_w, int64_t l) {
    float pmove = 3.0f / ((float)l + 3.0f);
    return wordify(scale_w, logf(pmove));
}

}  // namespace

struct cmgpu_vit_filter {
    int device = 0;
    VitHost host;
    int16_t *d_tab = nullptr;
    double last_ms = 0;
    int64_t last_cells = 0;
    cmx::DevArena arena;  // per-call buffers, reused
    ~cmgpu_vit_filter() {
        arena.release();
        cudaFree(d_tab);
    }
};

namespace cmx {
namespace dev {

__device__ __forceinline__ int adds16(int a, int b) {
    int s = a + b;
    return s > 32767 ? 32767 : (s < -32768 ? -32768 : s);
}

struct VitWin {
    int64_t off;    // frame offset in the residue buffer
    int32_t i0, j0; // residues scored: i0..j0
    int32_t xw_move;
    int32_t pad;
};

// One warp per window.  out[w] = final xC (int16 in an int32), status[w] =
// 1 scored, 0 overflow (xE reached 32767).  The score table is staged in
// shared memory transposed, tabT[c][k] (c = 0..25, k = 0..M), so the lanes
// of a warp read neighbouring positions of one entry.
__global__ void __launch_bounds__(256) vit_kernel(const int16_t *__restrict__ tab, int M, int base_w, int e_move,
                                                  int e_loop, const uint8_t *__restrict__ dsq,
                                                  const VitWin *__restrict__ wins, int nwin, int *out,
                                                  uint8_t *status) {
    extern __shared__ int vsm[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int B = (M + 31) / 32;
    const int stride = (B % 2 == 0) ? B + 1 : B + 2;  // odd stride: lanes hit distinct banks
    const int rowlen = 32 * stride;
    const int tstride = M + 2;                          // entries per table column (k = 0..M, padded)
    int16_t *tabT = reinterpret_cast<int16_t *>(vsm + (size_t)nw * 6 * rowlen);
    for (int q = threadIdx.x; q < (M + 1) * 26; q += blockDim.x) {
        const int k = q / 26, c = q - k * 26;
        tabT[c * tstride + k] = tab[q];
    }
    __syncthreads();
    auto T = [&](int c, int k) -> int { return tabT[c * tstride + k]; };
    int *base = vsm + (size_t)warp * 6 * rowlen;
    int *mp = base, *ip = base + rowlen, *dp = base + 2 * rowlen;
    int *mc = base + 3 * rowlen, *ic = base + 4 * rowlen, *dc = base + 5 * rowlen;
    const int k0 = 1 + lane * B;  // first position of this lane's block
    for (int w = blockIdx.x * nw + warp; w < nwin; w += gridDim.x * nw) {
        const VitWin win = wins[w];
        const uint8_t *frame = dsq + win.off;
        for (int b = 0; b < B; b++) {
            mp[lane * stride + b] = -32768;
            ip[lane * stride + b] = -32768;
            dp[lane * stride + b] = -32768;
        }
        int xn = base_w, xb = adds16(base_w, win.xw_move), xj = -32768, xc = -32768;
        bool overflow = false;
        __syncwarp();
        for (int i = win.i0; i <= win.j0; i++) {
            int x = frame[i];
            x = x > 17 ? 17 : x;
            // previous-row values at k0-1 (lane-1's last cell; -inf at k = 0)
            int pm = __shfl_up_sync(0xffffffffu, mp[lane * stride + B - 1], 1);
            int pi = __shfl_up_sync(0xffffffffu, ip[lane * stride + B - 1], 1);
            int pd = __shfl_up_sync(0xffffffffu, dp[lane * stride + B - 1], 1);
            if (lane == 0) pm = pi = pd = -32768;
            int xe = -32768;
            for (int b = 0; b < B; b++) {
                const int k = k0 + b;
                int vm = -32768, vi = -32768;
                if (k <= M) {
                    int sc = adds16(xb, T(18, k));
                    sc = max(sc, adds16(pm, T(19, k - 1)));
                    sc = max(sc, adds16(pi, T(20, k - 1)));
                    sc = max(sc, adds16(pd, T(21, k - 1)));
                    vm = adds16(sc, T(x, k));
                    const int cm = mp[lane * stride + b], ci = ip[lane * stride + b];
                    vi = max(adds16(cm, T(22, k)), adds16(ci, T(23, k)));
                    xe = max(xe, vm);
                }
                pm = mp[lane * stride + b];
                pi = ip[lane * stride + b];
                pd = dp[lane * stride + b];
                mc[lane * stride + b] = vm;
                ic[lane * stride + b] = vi;
            }
            for (int o = 16; o > 0; o >>= 1) xe = max(xe, __shfl_xor_sync(0xffffffffu, xe, o));
            __syncwarp();
            // D chain along k: d(k) = max(M(i,k-1)+MD(k-1), d(k-1)+DD(k-1))
            int m_in = __shfl_up_sync(0xffffffffu, mc[lane * stride + B - 1], 1);
            if (lane == 0) m_in = -32768;
            int din = -32768, din_prev = -32768;
            for (int it = 0; it < 34; it++) {
                int d = din, mprev = m_in;
                for (int b = 0; b < B; b++) {
                    const int k = k0 + b;
                    int v = -32768;
                    if (k <= M) v = max(adds16(mprev, T(24, k - 1)), adds16(d, T(25, k - 1)));
                    dc[lane * stride + b] = v;
                    d = v;
                    mprev = mc[lane * stride + b];
                }
                const bool has = k0 <= M;
                const int dlast = has ? d : -32768;
                const bool same = !has || din == din_prev;
                if (it > 0 && __all_sync(0xffffffffu, same)) break;
                din_prev = din;
                int up = __shfl_up_sync(0xffffffffu, dlast, 1);
                din = lane == 0 ? -32768 : up;
            }
            if (xe >= 32767) {
                overflow = true;
                break;
            }
            xc = max(xc, adds16(xe, e_move));
            xj = max(xj, adds16(xe, e_loop));
            xb = max(adds16(xj, win.xw_move), adds16(xn, win.xw_move));
            int *t;
            t = mp; mp = mc; mc = t;
            t = ip; ip = ic; ic = t;
            t = dp; dp = dc; dc = t;
            __syncwarp();
        }
        if (lane == 0) {
            out[w] = xc;
            status[w] = overflow ? 0 : 1;
        }
        __syncwarp();
        // keep the row roles fixed for the next window
        mp = base; ip = base + rowlen; dp = base + 2 * rowlen;
        mc = base + 3 * rowlen; ic = base + 4 * rowlen; dc = base + 5 * rowlen;
    }
}

// Packed kernel for models up to 256 positions: lane l owns the 2*NP
// positions k = 1 + 2*NP*l .. 2*NP*(l+1), held as NP registers of two int16
// cells each (the lower half is position k, the upper half k+1), for each of
// the M, I and D rows.  Every saturating step acts on two cells at once with
// the sm_90+ s16x2 instructions:
//   sat(a + b) = add(min(max(a, lo_b), hi_b), b),  lo_b = max(-32768 - b, -32768),
//                hi_b = min(32767 - b, 32767),
// which is exact: a is moved just far enough that a + b lands on the
// saturation bound, and otherwise left alone.  Transitions are never positive
// (they are capped at 0 or -1), so for them the upper clamp is the identity
// and only max + add remain.  The operations and their order per cell are
// those of the scalar recurrence, so the result is the same bit for bit.
__device__ __forceinline__ uint32_t pk16(int lo, int hi) { return ((uint32_t)lo & 0xffffu) | ((uint32_t)hi << 16); }
__device__ __forceinline__ int lo16(uint32_t x) { return (int)(int16_t)(x & 0xffffu); }
__device__ __forceinline__ int hi16(uint32_t x) { return (int)(int16_t)(x >> 16); }
__device__ __forceinline__ uint32_t vadd2(uint32_t a, uint32_t b) {
    uint32_t r;
    asm("add.s16x2 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
    return r;
}
__device__ __forceinline__ uint32_t vmax2(uint32_t a, uint32_t b) {
    uint32_t r;
    asm("max.s16x2 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
    return r;
}
__device__ __forceinline__ uint32_t vmin2(uint32_t a, uint32_t b) {
    uint32_t r;
    asm("min.s16x2 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
    return r;
}
// lower clamp of a non-positive addend: -32768 - b (b <= 0, so it fits)
__host__ __device__ __forceinline__ int lo_clamp(int b) { return b < 0 ? -32768 - b : -32768; }
__host__ __device__ __forceinline__ int hi_clamp(int b) { return b > 0 ? 32767 - b : 32767; }
// saturating add of a non-positive pair b, with lb its lower clamps
__device__ __forceinline__ uint32_t addsat_np(uint32_t a, uint32_t b, uint32_t lb) { return vadd2(vmax2(a, lb), b); }

template <int NP>
__global__ void __launch_bounds__(256) vit_kernel_pk(const int16_t *__restrict__ tab, int M, int base_w,
                                                     int e_move, int e_loop, const uint8_t *__restrict__ dsq,
                                                     const VitWin *__restrict__ wins, int nwin, int *out,
                                                     uint8_t *status) {
    // emission pairs [18][NP][32] as (b, lo_b, hi_b) triples, lane-minor so a
    // warp's reads of one entry hit 32 distinct banks
    extern __shared__ uint32_t psm[];
    constexpr int BB = 2 * NP;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    auto tv = [&](int k, int c) -> int { return (k >= 0 && k <= M) ? (int)tab[k * 26 + c] : -32768; };
    for (int q = threadIdx.x; q < 18 * NP * 32; q += blockDim.x) {
        const int x = q / (NP * 32), r = q - x * (NP * 32), qq = r >> 5, l = r & 31;
        const int k = 1 + l * BB + 2 * qq;
        const int a = tv(k, x), b = tv(k + 1, x);
        psm[3 * q] = pk16(a, b);
        psm[3 * q + 1] = pk16(lo_clamp(a), lo_clamp(b));
        psm[3 * q + 2] = pk16(hi_clamp(a), hi_clamp(b));
    }
    const int k0 = 1 + lane * BB;
    // transition pairs and their lower clamps; the ones read at k-1 are
    // stored shifted, (k-1, k) for the pair (k, k+1)
    uint32_t tb[NP], lb[NP], tmm[NP], lmm[NP], tim[NP], lim[NP], tdm[NP], ldm[NP];
    uint32_t tmi[NP], lmi[NP], tii[NP], lii[NP], tmd[NP], lmd[NP], tdd[NP], ldd[NP], inv[NP];
#pragma unroll
    for (int q = 0; q < NP; q++) {
        const int k = k0 + 2 * q;
#define VIT_PAIR(t, l, c, k1)                          \
    {                                                  \
        const int a_ = tv(k1, c), b_ = tv(k1 + 1, c);  \
        t[q] = pk16(a_, b_);                           \
        l[q] = pk16(lo_clamp(a_), lo_clamp(b_));       \
    }
        VIT_PAIR(tb, lb, 18, k)
        VIT_PAIR(tmm, lmm, 19, k - 1)
        VIT_PAIR(tim, lim, 20, k - 1)
        VIT_PAIR(tdm, ldm, 21, k - 1)
        VIT_PAIR(tmi, lmi, 22, k)
        VIT_PAIR(tii, lii, 23, k)
        VIT_PAIR(tmd, lmd, 24, k - 1)
        VIT_PAIR(tdd, ldd, 25, k - 1)
#undef VIT_PAIR
        inv[q] = (k > M ? 0x0000ffffu : 0u) | (k + 1 > M ? 0xffff0000u : 0u);
    }
    __syncthreads();
    const unsigned FULL = 0xffffffffu;
    const uint32_t NEG = 0x80008000u;
    for (int w = blockIdx.x * nw + warp; w < nwin; w += gridDim.x * nw) {
        const VitWin win = wins[w];
        const uint8_t *frame = dsq + win.off;
        uint32_t mv[NP], iv[NP], dv[NP];
#pragma unroll
        for (int q = 0; q < NP; q++) mv[q] = iv[q] = dv[q] = NEG;
        int xn = base_w, xb = adds16(base_w, win.xw_move), xj = -32768, xc = -32768;
        bool overflow = false;
        for (int i = win.i0; i <= win.j0; i++) {
            int x = frame[i];
            x = x > 17 ? 17 : x;
            const uint32_t *E = psm + 3 * (x * NP * 32 + lane);
            // previous-row cells at k0-1 (lane-1's last cell; -inf at k = 0)
            uint32_t pm = __shfl_up_sync(FULL, mv[NP - 1], 1);
            uint32_t pi = __shfl_up_sync(FULL, iv[NP - 1], 1);
            uint32_t pd = __shfl_up_sync(FULL, dv[NP - 1], 1);
            if (lane == 0) pm = pi = pd = NEG;
            const uint32_t XB = pk16(xb, xb);
            uint32_t mn[NP], in[NP], dn[NP], xe2 = NEG;
#pragma unroll
            for (int q = 0; q < NP; q++) {
                // previous row at (k-1, k): upper half of the pair before, lower half of this one
                const uint32_t sm = __byte_perm(pm, mv[q], 0x5432);
                const uint32_t si = __byte_perm(pi, iv[q], 0x5432);
                const uint32_t sd = __byte_perm(pd, dv[q], 0x5432);
                uint32_t sc = addsat_np(XB, tb[q], lb[q]);
                sc = vmax2(sc, addsat_np(sm, tmm[q], lmm[q]));
                sc = vmax2(sc, addsat_np(si, tim[q], lim[q]));
                sc = vmax2(sc, addsat_np(sd, tdm[q], ldm[q]));
                const uint32_t eb = E[96 * q], el = E[96 * q + 1], eh = E[96 * q + 2];
                uint32_t vm = vadd2(vmin2(vmax2(sc, el), eh), eb);
                uint32_t vi = vmax2(addsat_np(mv[q], tmi[q], lmi[q]), addsat_np(iv[q], tii[q], lii[q]));
                vm = (vm & ~inv[q]) | (NEG & inv[q]);
                vi = (vi & ~inv[q]) | (NEG & inv[q]);
                xe2 = vmax2(xe2, vm);
                pm = mv[q];
                pi = iv[q];
                pd = dv[q];
                mn[q] = vm;
                in[q] = vi;
            }
            int xe = max(lo16(xe2), hi16(xe2));
            for (int o = 16; o > 0; o >>= 1) xe = max(xe, __shfl_xor_sync(FULL, xe, o));
            // D chain along k: d(k) = max(M(i,k-1)+MD(k-1), d(k-1)+DD(k-1));
            // the M terms of every pair first (independent of d), then the chain
            uint32_t m_in = __shfl_up_sync(FULL, mn[NP - 1], 1);
            if (lane == 0) m_in = NEG;
            uint32_t mt[NP];
#pragma unroll
            for (int q = 0; q < NP; q++) {
                const uint32_t smn = __byte_perm(q == 0 ? m_in : mn[q > 0 ? q - 1 : 0], mn[q], 0x5432);
                mt[q] = addsat_np(smn, tmd[q], lmd[q]);
            }
            int din = -32768, din_prev = -32768;
            for (int it = 0; it < 34; it++) {
                uint32_t d = pk16(din, din);  // the chain value in both halves
#pragma unroll
                for (int q = 0; q < NP; q++) {
                    const uint32_t r1 = vmax2(mt[q], addsat_np(d, tdd[q], ldd[q]));   // lower half: d(k)
                    const uint32_t d1 = __byte_perm(r1, 0, 0x1010);
                    const uint32_t r2 = vmax2(mt[q], addsat_np(d1, tdd[q], ldd[q]));  // upper half: d(k+1)
                    uint32_t v = __byte_perm(r1, r2, 0x7610);
                    v = (v & ~inv[q]) | (NEG & inv[q]);
                    dn[q] = v;
                    d = __byte_perm(v, 0, 0x3232);
                }
                const bool has = k0 <= M;
                const int dlast = has ? hi16(d) : -32768;
                const bool same = !has || din == din_prev;
                if (it > 0 && __all_sync(FULL, same)) break;
                din_prev = din;
                const int up = __shfl_up_sync(FULL, dlast, 1);
                din = lane == 0 ? -32768 : up;
            }
            if (xe >= 32767) {
                overflow = true;
                break;
            }
            xc = max(xc, adds16(xe, e_move));
            xj = max(xj, adds16(xe, e_loop));
            xb = max(adds16(xj, win.xw_move), adds16(xn, win.xw_move));
#pragma unroll
            for (int q = 0; q < NP; q++) {
                mv[q] = mn[q];
                iv[q] = in[q];
                dv[q] = dn[q];
            }
        }
        if (lane == 0) {
            out[w] = xc;
            status[w] = overflow ? 0 : 1;
        }
    }
}

}  // namespace dev
}  // namespace cmx

using namespace cmx;

#define VIT_TRY(call)                                                                           \
    do {                                                                                        \
        cudaError_t e_ = (call);                                                                \
        if (e_ != cudaSuccess) {                                                                \
            set_error(std::string(#call) + ": " + cudaGetErrorString(e_));                      \
            return CMGPU_EDEVICE;                                                               \
        }                                                                                       \
    } while (0)

extern "C" int cmgpu_vit_filter_build(const cmgpu_p7_profile *p, int device, cmgpu_vit_filter **out) {
    if (!p || !out) return CMGPU_EINVAL;
    *out = nullptr;
    std::unique_ptr<cmgpu_vit_filter> f(new cmgpu_vit_filter());
    f->device = device;
    if (!build_vit(p, f->host)) {
        set_error("cmgpu_vit_filter_build: bad profile");
        return CMGPU_EINVAL;
    }
    if (device >= 0) {  // device < 0: host tables only (no GPU needed)
        VIT_TRY(cudaSetDevice(device));
        VIT_TRY(cudaMalloc((void **)&f->d_tab, f->host.tab.size() * sizeof(int16_t)));
        VIT_TRY(cudaMemcpy(f->d_tab, f->host.tab.data(), f->host.tab.size() * sizeof(int16_t),
                           cudaMemcpyHostToDevice));
    }
    *out = f.release();
    return CMGPU_OK;
}

extern "C" void cmgpu_vit_filter_free(cmgpu_vit_filter *f) { delete f; }

extern "C" int cmgpu_vit_filter_tables(const cmgpu_vit_filter *f, int16_t *tab, int32_t cap, int32_t *n_out,
                                       int16_t *specials) {
    if (!f || !n_out) return CMGPU_EINVAL;
    *n_out = (int32_t)f->host.tab.size();
    if (specials) {
        specials[0] = f->host.base_w;
        specials[1] = f->host.e_move;
        specials[2] = f->host.e_loop;
    }
    if ((int64_t)f->host.tab.size() > cap) return CMGPU_EOVERFLOW;
    if (tab) std::copy(f->host.tab.begin(), f->host.tab.end(), tab);
    return CMGPU_OK;
}

extern "C" int cmgpu_vit_score_batch(const cmgpu_vit_filter *f, void *stream_ptr, const uint8_t *dsq_all,
                                     int64_t dsq_len, const cmgpu_window *wins, int32_t nwin, float *scores,
                                     uint8_t *scored) {
    if (!f || !dsq_all || nwin < 0 || (nwin > 0 && (!wins || !scores || !scored))) return CMGPU_EINVAL;
    if (!f->d_tab) {
        set_error("cmgpu_vit_score_batch: filter was built without a device");
        return CMGPU_EINVAL;
    }
    if (nwin == 0) return CMGPU_OK;
    std::vector<dev::VitWin> vw(nwin);
    for (int32_t k = 0; k < nwin; k++) {
        const cmgpu_window &w = wins[k];
        if (w.dsq_offset < 0 || w.i0 < 1 || w.j0 < w.i0 - 1 || w.dsq_offset + (int64_t)w.j0 + 1 > dsq_len) {
            set_error("cmgpu_vit_score_batch: window outside the residue buffer");
            return CMGPU_EINVAL;
        }
        if (w.j0 >= w.i0 && cmx::any_code_above_17(dsq_all + w.dsq_offset + w.i0, (int64_t)w.j0 - w.i0 + 1)) {
            set_error("cmgpu_vit_score_batch: residue code > 17");
            return CMGPU_EINVAL;
        }
        vw[k].off = w.dsq_offset;
        vw[k].i0 = w.i0;
        vw[k].j0 = w.j0;
        vw[k].xw_move = xw_move_for(f->host.scale_w, (int64_t)w.j0 - w.i0 + 1);
        vw[k].pad = 0;
    }
    cudaStream_t st = (cudaStream_t)stream_ptr;
    VIT_TRY(cudaSetDevice(f->device));
    uint8_t *d_dsq = nullptr;
    dev::VitWin *d_w = nullptr;
    int *d_out = nullptr;
    uint8_t *d_st = nullptr;
    cmgpu_vit_filter *mf = const_cast<cmgpu_vit_filter *>(f);
    auto cleanup = [&]() {};
    cudaError_t e = cudaSuccess;
    if ((e = mf->arena.get(0, &d_dsq, (size_t)dsq_len)) != cudaSuccess ||
        (e = mf->arena.get(1, &d_w, sizeof(dev::VitWin) * nwin)) != cudaSuccess ||
        (e = mf->arena.get(2, &d_out, sizeof(int) * nwin)) != cudaSuccess ||
        (e = mf->arena.get(3, &d_st, (size_t)nwin)) != cudaSuccess) {
        cleanup();
        set_error(std::string("cmgpu_vit_score_batch: ") + cudaGetErrorString(e));
        return CMGPU_ENOMEM;
    }
    const int M = f->host.M;
    const int B = (M + 31) / 32;
    const int stride = (B % 2 == 0) ? B + 1 : B + 2;
    const size_t tab_bytes = ((size_t)26 * (M + 2) * sizeof(int16_t) + 15) & ~(size_t)15;
    int warps = 8;
    size_t smem = (size_t)warps * 6 * 32 * stride * sizeof(int) + tab_bytes;
    while (smem > 200 * 1024 && warps > 1) {
        warps /= 2;
        smem = (size_t)warps * 6 * 32 * stride * sizeof(int) + tab_bytes;
    }
    if (smem > 227 * 1024) {
        cleanup();
        set_error("cmgpu_vit_score_batch: model too long for the shared-memory rows");
        return CMGPU_ENOSPACE;
    }
    std::vector<int> out(nwin);
    std::vector<uint8_t> stv(nwin);
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, f->device);
    int grid = (int)std::min<int64_t>((nwin + warps - 1) / warps, (int64_t)sms * 8);
    if ((e = cudaMemcpyAsync(d_dsq, dsq_all, (size_t)dsq_len, cudaMemcpyHostToDevice, st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(d_w, vw.data(), sizeof(dev::VitWin) * nwin, cudaMemcpyHostToDevice, st)) !=
            cudaSuccess ||
        (e = cmx::allow_max_dynamic_smem(dev::vit_kernel)) !=
            cudaSuccess) {
        cleanup();
        set_error(std::string("cmgpu_vit_score_batch: ") + cudaGetErrorString(e));
        return CMGPU_EDEVICE;
    }
    // models up to 256 positions keep each lane's block of the rows in
    // registers as packed int16 pairs; longer ones use the shared-memory rows
    const int NP = (B + 1) / 2;
    auto launch_pk = [&](auto kern) {
        const int g = (int)std::min<int64_t>((nwin + 7) / 8, (int64_t)sms * 8);
        const size_t pk_smem = (size_t)18 * NP * 32 * 3 * sizeof(uint32_t);
        cmx::allow_max_dynamic_smem(kern);
        kern<<<g, 256, pk_smem, st>>>(f->d_tab, M, f->host.base_w, f->host.e_move, f->host.e_loop, d_dsq, d_w,
                                      nwin, d_out, d_st);
    };
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaEventCreate(&ev0);
    cudaEventCreate(&ev1);
    cudaEventRecord(ev0, st);
    switch (B <= 8 ? NP : 0) {
    case 1: launch_pk(dev::vit_kernel_pk<1>); break;
    case 2: launch_pk(dev::vit_kernel_pk<2>); break;
    case 3: launch_pk(dev::vit_kernel_pk<3>); break;
    case 4: launch_pk(dev::vit_kernel_pk<4>); break;
    default:
        dev::vit_kernel<<<grid, warps * 32, smem, st>>>(f->d_tab, M, f->host.base_w, f->host.e_move, f->host.e_loop,
                                                      d_dsq, d_w, nwin, d_out, d_st);
    }
    cudaEventRecord(ev1, st);
    if ((e = cudaGetLastError()) != cudaSuccess ||
        (e = cudaMemcpyAsync(out.data(), d_out, sizeof(int) * nwin, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(stv.data(), d_st, (size_t)nwin, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess) {
        cleanup();
        cudaEventDestroy(ev0);
        cudaEventDestroy(ev1);
        set_error(std::string("cmgpu_vit_score_batch: ") + cudaGetErrorString(e));
        return CMGPU_EDEVICE;
    }
    cleanup();
    {
        float ms = 0;
        cudaEventElapsedTime(&ms, ev0, ev1);
        cudaEventDestroy(ev0);
        cudaEventDestroy(ev1);
        mf->last_ms = ms;
        mf->last_cells = 0;
        for (int32_t k = 0; k < nwin; k++) mf->last_cells += (int64_t)(wins[k].j0 - wins[k].i0 + 1) * M;
    }
    // C->T (src/p7_vitfilter.rs:376-384), in f32 as the reference
    for (int32_t k = 0; k < nwin; k++) {
        scored[k] = stv[k];
        if (!stv[k]) {
            scores[k] = NAN;
            continue;
        }
        int xc = out[k];
        if (xc > -32768) {
            float ret = (float)xc + (float)vw[k].xw_move - (float)f->host.base_w;
            ret /= f->host.scale_w;
            scores[k] = ret - 3.0f;
        } else {
            scores[k] = -INFINITY;
        }
    }
    return CMGPU_OK;
}

extern "C" int cmgpu_vit_filter_stats(const cmgpu_vit_filter *f, double *kernel_ms, int64_t *cells,
                                      int32_t *launches) {
    if (!f) return CMGPU_EINVAL;
    if (kernel_ms) *kernel_ms = f->last_ms;
    if (cells) *cells = f->last_cells;
    if (launches) *launches = f->last_ms > 0 ? 1 : 0;
    return CMGPU_OK;
}
