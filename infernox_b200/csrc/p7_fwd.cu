// P7 local Forward filter (F3), composition-bias filter (F3b) and the F1 ->
// F3b window cascade of one pipeline pass.
//
// Host side: the odds-space profile is built as the reference builds it
// (build_forward_filter, src/cm_pipeline.rs:969-1120): match odds exp(ln(p /
// 0.25)) with IUPAC codes the mean of their residues' log-odds, local entries
// from the match occupancy round-tripped through log / exp, and the raw
// transitions; then packed in the striped order of the reference's default
// engine (forward_filter_score_striped, :1270-1418): nq = max(2, (M-1)/4+1)
// vectors of four lanes, cell (q, z) = model position q + 1 + z * nq, zero
// beyond M.  The bias filter is the two-state null of build_bias_filter
// (:1683-1720).
//
// Device side, Forward: four threads per window, thread z playing lane z of
// the reference's 128-bit vectors.  A lane's cells are the contiguous model
// positions z*nq+1 .. (z+1)*nq, so each thread walks its own segment in q
// order, and the only cross-lane steps -- the shift that feeds a segment's
// first cell from the previous segment's last, and the final horizontal sum
// of xE -- are shuffles inside the group of four.  Every multiply and add is
// rounded on its own (-fmad=false) in the reference's order: per-lane xE
// accumulation over q, the obligatory D pass plus three more (all three for
// M < 100, stopping at the first pass that changes no cell of the group for
// M >= 100), the horizontal sum (x0 + x1) + (x2 + x3), the N/C/J/B specials
// and the sparse rescaling at xE > 1e4, whose logarithm is taken in double
// precision.  Models with nq <= 32 keep a lane's segment of the window's M,
// D and I rows in registers (fwd_kernel_reg); longer ones keep the rows in
// shared memory, each group at a stride of 4 (mod 32) words so that the 32
// threads of a warp touch 32 banks (fwd_kernel).  Groups take windows from a
// device counter, longest first.  A D pass "changes" a cell when its bits
// change: D values are sums of products of probabilities, never negative,
// so that is the reference's d > old.
//
// Device side, bias: one thread per window, the two-state forward with
// per-row max rescaling (:1722-1790), on a second stream of the filter so it
// runs beside the Forward kernel; the length term is added on the host
// (glibc logf, as the reference).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <utility>
#include <string>
#include <vector>

#include "../../include/cmscan_gpu.h"
#include "devbuf.h"

namespace cmx {
void set_error(const std::string &msg);
int f1_msv_windows_vec(const cmgpu_msv_filter *f, cudaStream_t st, const uint8_t *dsq_all, int64_t dsq_len,
                       const cmgpu_window *chunks, int32_t nchunk, double f1, int64_t cmw,
                       std::vector<cmgpu_f1_window> &wins);
}
using cmx::set_error;

namespace {

constexpr int KP = 18;
constexpr int KC = 4;

// canonical residues of each RNA code (src/cm_pipeline.rs:129-155)
const int DEGEN[KP][5] = {
    {1, 0}, {1, 1}, {1, 2}, {1, 3}, {0},      {2, 0, 2}, {2, 1, 3}, {2, 0, 1}, {2, 2, 3},
    {2, 1, 2}, {2, 0, 3}, {3, 0, 1, 3}, {3, 1, 2, 3}, {3, 0, 1, 2}, {3, 0, 2, 3}, {4, 0, 1, 2, 3}, {0}, {0}};

// striped table rows per vector q: the seven main transitions in the
// reference's order, then DD
enum { T_BM, T_MM, T_IM, T_DM, T_MD, T_MI, T_II, T_DD, T_N };

struct FwdHost {
    int M = 0, nq = 2, rq = 3;
    std::vector<float> rfv;   // [(M+1)][KP] match odds, natural order
    std::vector<float> tr;    // [(M+1)][8]: tbm, amm, aim, adm, tmi, tii, tmd, tdd
    std::vector<float> stab;  // device layout: [nq][T_N][4], then rfv [KP][rq][4]
    std::vector<float> ptab;  // register kernel: [nq][4][T_N] (a lane's eight values together), then rfv as above
    float eo[KP * 2] = {};
    float t1[3] = {};
    double ftau = 0, flambda = 0;
};

void build_host(const cmgpu_p7_profile *p, const float *compo, FwdHost &h) {
    const int m = p->M;
    h.M = m;
    h.nq = std::max(2, m >= 1 ? (m - 1) / 4 + 1 : 2);
    h.rq = h.nq | 1;  // odd row stride: residue rows of different codes fall in different banks
    h.rfv.assign((size_t)(m + 1) * KP, 0.0f);
    h.tr.assign((size_t)(m + 1) * 8, 0.0f);
    for (int k = 1; k <= m; k++) {
        float sc[KP];
        for (int x = 0; x < KP; x++) sc[x] = -INFINITY;
        for (int x = 0; x < KC; x++) sc[x] = (float)std::log((double)p->mat[k * 4 + x] / 0.25);
        for (int code = KC; code < KP; code++) {
            const int n = DEGEN[code][0];
            if (n == 0) continue;
            float s = 0.0f;
            for (int q = 0; q < n; q++) s += sc[DEGEN[code][1 + q]];
            sc[code] = s / (float)n;
        }
        for (int x = 0; x < KP; x++) h.rfv[(size_t)k * KP + x] = std::exp(sc[x]);  // expf
    }
    // match occupancy and local entries (src/cm_pipeline.rs:1013-1040)
    const float *t = p->trans;
    std::vector<float> occ(m + 1, 0.0f);
    if (m >= 1) occ[1] = t[1] + t[0];
    for (int k = 2; k <= m; k++)
        occ[k] = occ[k - 1] * (t[(k - 1) * 7 + 0] + t[(k - 1) * 7 + 1]) + (1.0f - occ[k - 1]) * t[(k - 1) * 7 + 5];
    float z = 0.0f;
    for (int k = 1; k <= m; k++) z += occ[k] * (float)(m - k + 1);
    auto TR = [&](int k, int a) -> float & { return h.tr[(size_t)k * 8 + a]; };
    for (int k = 1; k <= m; k++) {
        TR(k, 0) = (float)std::exp(std::log((double)(occ[k] / z)));
        TR(k, 1) = t[(k - 1) * 7 + 0];  // M(k-1) -> M(k)
        TR(k, 2) = t[(k - 1) * 7 + 3];  // I(k-1) -> M(k)
        TR(k, 3) = t[(k - 1) * 7 + 5];  // D(k-1) -> M(k)
    }
    for (int k = 1; k < m; k++) {
        TR(k, 4) = t[k * 7 + 1];  // M -> I
        TR(k, 5) = t[k * 7 + 4];  // I -> I
        TR(k, 6) = t[k * 7 + 2];  // M -> D(k+1)
        TR(k, 7) = t[k * 7 + 6];  // D -> D(k+1)
    }
    // striped packing
    const int nq = h.nq, rq = h.rq;
    h.stab.assign((size_t)nq * T_N * 4 + (size_t)KP * rq * 4, 0.0f);
    static const int SRC[T_N] = {0, 1, 2, 3, 6, 4, 5, 7};  // striped row -> natural column
    for (int q = 0; q < nq; q++)
        for (int zz = 0; zz < 4; zz++) {
            const int pos = q + 1 + zz * nq;
            if (pos > m) continue;
            for (int r = 0; r < T_N; r++) h.stab[((size_t)q * T_N + r) * 4 + zz] = TR(pos, SRC[r]);
            for (int x = 0; x < KP; x++)
                h.stab[(size_t)nq * T_N * 4 + ((size_t)x * rq + q) * 4 + zz] = h.rfv[(size_t)pos * KP + x];
        }
    h.ptab.assign(h.stab.size(), 0.0f);
    for (int q = 0; q < nq; q++)
        for (int zz = 0; zz < 4; zz++)
            for (int r = 0; r < T_N; r++)
                h.ptab[((size_t)q * 4 + zz) * T_N + r] = h.stab[((size_t)q * T_N + r) * 4 + zz];
    std::copy(h.stab.begin() + (size_t)nq * T_N * 4, h.stab.end(), h.ptab.begin() + (size_t)nq * T_N * 4);
    // bias filter (src/cm_pipeline.rs:1683-1720)
    const float bg = 0.25f;
    const float l1 = (float)m / 8.0f;
    for (int code = 0; code < KP; code++) {
        h.eo[code * 2 + 0] = 1.0f;
        const int n = DEGEN[code][0];
        if (n == 0) {
            h.eo[code * 2 + 1] = 1.0f;
            continue;
        }
        float num = 0.0f, den = 0.0f;
        for (int q = 0; q < n; q++) {
            num += compo[DEGEN[code][1 + q]];
            den += bg;
        }
        h.eo[code * 2 + 1] = den > 0.0f ? num / den : 0.0f;
    }
    h.t1[0] = 1.0f / (l1 + 1.0f);
    h.t1[1] = l1 / (l1 + 1.0f);
    h.t1[2] = 1.0f;
}

}  // namespace

struct cmgpu_fwd_filter {
    int device = 0;
    FwdHost host;
    float *d_tab = nullptr;
    float *d_ptab = nullptr;
    int kernel = CMGPU_FWD_KERNEL_AUTO;
    cudaStream_t side = nullptr;  // the bias kernel runs here, beside the Forward kernel
    cudaEvent_t fork = nullptr, join = nullptr;
    cudaEvent_t t0 = nullptr, t1 = nullptr;  // device time of a call
    double last_ms = 0;
    int64_t last_cells = 0;
    int32_t last_launches = 0;
    cmx::DevArena arena;  // per-call buffers, reused
    ~cmgpu_fwd_filter() {
        arena.release();
        cudaFree(d_tab);
        cudaFree(d_ptab);
        if (fork) cudaEventDestroy(fork);
        if (join) cudaEventDestroy(join);
        if (t0) cudaEventDestroy(t0);
        if (t1) cudaEventDestroy(t1);
        if (side) cudaStreamDestroy(side);
    }
};

namespace cmx {
namespace dev {

struct FwdWin {
    int64_t first;  // offset of residue 1 of the window in the residue buffer
    int32_t L;
    int32_t pad;
};

struct BiasParams {
    float eo[KP * 2];
    float t1[3];
};

// value of lane z-1 of the group of four; zero for lane 0 (the reference's
// byte shift of a vector by one float)
__device__ __forceinline__ float lane_shift(unsigned gmask, float v, int z) {
    const float t = __shfl_up_sync(gmask, v, 1, 4);
    return z == 0 ? 0.0f : t;
}

// Forward score pieces of each window: (total of the rescaling logs, xC).
// TS: the striped tables are staged in shared memory.
template <bool TS>
__global__ void __launch_bounds__(256) fwd_kernel(const float *__restrict__ tab, int M, int nq, int rq, int gstride,
                                                  const uint8_t *__restrict__ dsq, const FwdWin *__restrict__ wins,
                                                  int nwin, int *__restrict__ next, float2 *__restrict__ out) {
    extern __shared__ __align__(16) float sm[];
    const int tabn = nq * T_N * 4 + KP * rq * 4;
    const float *T = tab;
    float *state = sm;
    if (TS) {
        for (int q = threadIdx.x; q < tabn; q += blockDim.x) sm[q] = tab[q];
        __syncthreads();
        T = sm;
        state = sm + ((tabn + 31) & ~31);
    }
    const int lane = threadIdx.x & 31, z = lane & 3;
    const unsigned gmask = 0xFu << (lane & ~3);
    float *mmr = state + (threadIdx.x >> 2) * gstride;
    float *dmr = mmr + nq * 4;
    float *imr = dmr + nq * 4;
    const float *R0 = T + nq * T_N * 4;
    const bool lazy = M >= 100;
    for (;;) {
        int w = 0;
        if (z == 0) w = atomicAdd(next, 1);
        w = __shfl_sync(gmask, w, lane & ~3);
        if (w >= nwin) break;
        const FwdWin win = wins[w];
        const uint8_t *d = dsq + win.first - 1;
        const int L = win.L;
        for (int q = 0; q < nq; q++) {
            mmr[q * 4 + z] = 0.0f;
            dmr[q * 4 + z] = 0.0f;
            imr[q * 4 + z] = 0.0f;
        }
        const float pmove = 3.0f / ((float)L + 2.0f + 1.0f);
        const float ploop = 1.0f - pmove;
        float xn = 1.0f, xj = 0.0f, xb = pmove, xc = 0.0f, tot = 0.0f;
        for (int i = 1; i <= L; i++) {
            const float *rf = R0 + (int)d[i] * rq * 4;
            float mpv = lane_shift(gmask, mmr[(nq - 1) * 4 + z], z);
            float dpv = lane_shift(gmask, dmr[(nq - 1) * 4 + z], z);
            float ipv = lane_shift(gmask, imr[(nq - 1) * 4 + z], z);
            float dcv = 0.0f, xev = 0.0f;
            for (int q = 0; q < nq; q++) {
                const float *tq = T + q * (T_N * 4) + z;
                float sv = xb * tq[T_BM * 4];
                sv = sv + mpv * tq[T_MM * 4];
                sv = sv + ipv * tq[T_IM * 4];
                sv = sv + dpv * tq[T_DM * 4];
                sv = sv * rf[q * 4 + z];
                xev = xev + sv;
                mpv = mmr[q * 4 + z];
                dpv = dmr[q * 4 + z];
                ipv = imr[q * 4 + z];
                mmr[q * 4 + z] = sv;
                dmr[q * 4 + z] = dcv;
                dcv = sv * tq[T_MD * 4];
                imr[q * 4 + z] = mpv * tq[T_MI * 4] + ipv * tq[T_II * 4];
            }
            // D paths: the obligatory pass, then up to three more
            dcv = lane_shift(gmask, dcv, z);
            dmr[z] = 0.0f;
            for (int q = 0; q < nq; q++) {
                const float dd = dcv + dmr[q * 4 + z];
                dmr[q * 4 + z] = dd;
                dcv = dd * T[q * (T_N * 4) + T_DD * 4 + z];
            }
            for (int j = 1; j < 4; j++) {
                dcv = lane_shift(gmask, dcv, z);
                int changed = 0;
                for (int q = 0; q < nq; q++) {
                    const float old = dmr[q * 4 + z];
                    const float dd = dcv + old;
                    changed |= __float_as_int(dd) ^ __float_as_int(old);  // dcv >= 0: differs iff dd > old
                    dmr[q * 4 + z] = dd;
                    dcv = dcv * T[q * (T_N * 4) + T_DD * 4 + z];
                }
                if (lazy) {
                    changed |= __shfl_xor_sync(gmask, changed, 1, 4);
                    changed |= __shfl_xor_sync(gmask, changed, 2, 4);
                    if (!changed) break;
                }
            }
            for (int q = 0; q < nq; q++) xev = xev + dmr[q * 4 + z];
            // horizontal sum (x0 + x1) + (x2 + x3)
            const float h = xev + __shfl_sync(gmask, xev, (z + 1) & 3, 4);
            const float xe = __shfl_sync(gmask, h, 0, 4) + __shfl_sync(gmask, h, 2, 4);
            xn = xn * ploop;
            xc = (xc * ploop) + (xe * 0.5f);
            xj = (xj * ploop) + (xe * 0.5f);
            xb = (xj * pmove) + (xn * pmove);
            if (xe > 1.0e4f) {
                const float inv = __fdiv_rn(1.0f, xe);
                xn *= inv;
                xc *= inv;
                xj *= inv;
                xb *= inv;
                for (int q = 0; q < nq; q++) {
                    mmr[q * 4 + z] *= inv;
                    dmr[q * 4 + z] *= inv;
                    imr[q * 4 + z] *= inv;
                }
                tot += (float)log((double)xe);
            }
        }
        if (z == 0) out[w] = make_float2(tot, xc);
    }
}

// The same recurrence with a lane's segment of the M, D and I rows in
// registers: NQ = nq exactly (one instantiation per segment length, so no
// cell needs a bounds test), the lane's seven transition values of a cell
// read from shared memory as two 16-byte words, D->D read per pass.  LAZY:
// M >= 100, the D passes stop at the first one that changes no cell.
template <int NQ, bool LAZY>
__global__ void __launch_bounds__(128, 3) fwd_kernel_reg(const float *__restrict__ ptab, int rq,
                                                      const uint8_t *__restrict__ dsq,
                                                      const FwdWin *__restrict__ wins, int nwin,
                                                      int *__restrict__ next, float2 *__restrict__ out) {
    extern __shared__ __align__(16) float sm[];
    const int tabn = NQ * T_N * 4 + KP * rq * 4;
    for (int q = threadIdx.x; q < tabn; q += blockDim.x) sm[q] = ptab[q];
    __syncthreads();
    const int lane = threadIdx.x & 31, z = lane & 3;
    const unsigned gmask = 0xFu << (lane & ~3);
    const float4 *T4 = reinterpret_cast<const float4 *>(sm) + z * 2;
    const float *TD = sm + z * T_N + T_DD;
    const float *R0 = sm + NQ * T_N * 4 + z;
    float mmv[NQ], dmv[NQ], imv[NQ];
    for (;;) {
        int w = 0;
        if (z == 0) w = atomicAdd(next, 1);
        w = __shfl_sync(gmask, w, lane & ~3);
        if (w >= nwin) break;
        const FwdWin win = wins[w];
        const uint8_t *d = dsq + win.first - 1;
        const int L = win.L;
#pragma unroll
        for (int q = 0; q < NQ; q++) mmv[q] = dmv[q] = imv[q] = 0.0f;
        const float pmove = 3.0f / ((float)L + 2.0f + 1.0f);
        const float ploop = 1.0f - pmove;
        float xn = 1.0f, xj = 0.0f, xb = pmove, xc = 0.0f, tot = 0.0f;
        for (int i = 1; i <= L; i++) {
            const float *rf = R0 + (int)d[i] * rq * 4;
            float mpv = lane_shift(gmask, mmv[NQ - 1], z);
            float dpv = lane_shift(gmask, dmv[NQ - 1], z);
            float ipv = lane_shift(gmask, imv[NQ - 1], z);
            float dcv = 0.0f, xev = 0.0f;
#pragma unroll
            for (int q = 0; q < NQ; q++) {
                const float4 ta = T4[q * 8], tb = T4[q * 8 + 1];
                float sv = xb * ta.x;
                sv = sv + mpv * ta.y;
                sv = sv + ipv * ta.z;
                sv = sv + dpv * ta.w;
                sv = sv * rf[q * 4];
                xev = xev + sv;
                mpv = mmv[q];
                dpv = dmv[q];
                ipv = imv[q];
                mmv[q] = sv;
                dmv[q] = dcv;
                dcv = sv * tb.x;
                imv[q] = mpv * tb.y + ipv * tb.z;
            }
            dcv = lane_shift(gmask, dcv, z);
            dmv[0] = 0.0f;
#pragma unroll
            for (int q = 0; q < NQ; q++) {
                const float dd = dcv + dmv[q];
                dmv[q] = dd;
                dcv = dd * TD[q * 32];
            }
            for (int j = 1; j < 4; j++) {
                dcv = lane_shift(gmask, dcv, z);
                int changed = 0;
#pragma unroll
                for (int q = 0; q < NQ; q++) {
                    const float old = dmv[q];
                    const float dd = dcv + old;
                    if (LAZY) changed |= __float_as_int(dd) ^ __float_as_int(old);
                    dmv[q] = dd;
                    dcv = dcv * TD[q * 32];
                }
                if (LAZY) {
                    changed |= __shfl_xor_sync(gmask, changed, 1, 4);
                    changed |= __shfl_xor_sync(gmask, changed, 2, 4);
                    if (!changed) break;
                }
            }
#pragma unroll
            for (int q = 0; q < NQ; q++) xev = xev + dmv[q];
            const float h = xev + __shfl_sync(gmask, xev, (z + 1) & 3, 4);
            const float xe = __shfl_sync(gmask, h, 0, 4) + __shfl_sync(gmask, h, 2, 4);
            xn = xn * ploop;
            xc = (xc * ploop) + (xe * 0.5f);
            xj = (xj * ploop) + (xe * 0.5f);
            xb = (xj * pmove) + (xn * pmove);
            if (xe > 1.0e4f) {
                const float inv = __fdiv_rn(1.0f, xe);
                xn *= inv;
                xc *= inv;
                xj *= inv;
                xb *= inv;
#pragma unroll
                for (int q = 0; q < NQ; q++) {
                    mmv[q] *= inv;
                    dmv[q] *= inv;
                    imv[q] *= inv;
                }
                tot += (float)log((double)xe);
            }
        }
        if (z == 0) out[w] = make_float2(tot, xc);
    }
}

typedef void (*FwdRegFn)(const float *, int, const uint8_t *, const FwdWin *, int, int *, float2 *);

// the register kernel for segment length nq (2..32) and the D-pass rule
template <int... Q>
FwdRegFn fwd_reg_kernel(int nq, bool lazy, std::integer_sequence<int, Q...>) {
    static const FwdRegFn fixed[] = {fwd_kernel_reg<Q + 2, false>...};
    static const FwdRegFn early[] = {fwd_kernel_reg<Q + 2, true>...};
    return (lazy ? early : fixed)[nq - 2];
}

// bias_filter_score before its length term, one thread per window
__global__ void bias_kernel(BiasParams bp, const uint8_t *__restrict__ dsq, const FwdWin *__restrict__ wins, int nwin,
                            float *__restrict__ rows) {
    const int w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= nwin) return;
    const FwdWin win = wins[w];
    const int L = win.L;
    if (L == 0) {
        rows[w] = 0.0f;
        return;
    }
    const uint8_t *d = dsq + win.first - 1;
    const float lf = (float)L;
    const float p1 = __fdiv_rn(lf, lf + 1.0f);
    const float t00 = p1, t01 = 1.0f - p1;
    const float t10 = bp.t1[0], t11 = bp.t1[1];
    int x = d[1];
    float dp0 = bp.eo[x * 2 + 0] * 0.999f, dp1 = bp.eo[x * 2 + 1] * 0.001f;
    float mx = fmaxf(dp0, dp1);
    dp0 = __fdiv_rn(dp0, mx);
    dp1 = __fdiv_rn(dp1, mx);
    float logsc = (float)log((double)mx);
    for (int i = 2; i <= L; i++) {
        x = d[i];
        float s0 = 0.0f;
        s0 += dp0 * t00;
        s0 += dp1 * t10;
        float s1 = 0.0f;
        s1 += dp0 * t01;
        s1 += dp1 * t11;
        const float n0 = s0 * bp.eo[x * 2 + 0], n1 = s1 * bp.eo[x * 2 + 1];
        mx = fmaxf(n0, n1);
        dp0 = __fdiv_rn(n0, mx);
        dp1 = __fdiv_rn(n1, mx);
        logsc += (float)log((double)mx);
    }
    const float end = dp0 * 1.0f + dp1 * bp.t1[2];
    logsc += (float)log((double)end);
    rows[w] = logsc;
}

}  // namespace dev
}  // namespace cmx

namespace {

#define FWD_TRY(call)                                                                          \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess) {                                                               \
            set_error(std::string("fwd: ") + #call + ": " + cudaGetErrorString(e_));           \
            return CMGPU_EDEVICE;                                                              \
        }                                                                                      \
    } while (0)

int check_windows(const char *who, const uint8_t *dsq_all, int64_t dsq_len, const cmgpu_window *wins, int32_t nwin) {
    for (int32_t k = 0; k < nwin; k++) {
        const cmgpu_window &w = wins[k];
        if (w.dsq_offset < 0 || w.i0 < 1 || w.j0 < w.i0 - 1 || w.dsq_offset + (int64_t)w.j0 + 1 > dsq_len) {
            set_error(std::string(who) + ": window outside the residue buffer");
            return CMGPU_EINVAL;
        }
        if (w.j0 >= w.i0 && cmx::any_code_above_17(dsq_all + w.dsq_offset + w.i0, (int64_t)w.j0 - w.i0 + 1)) {
            set_error(std::string(who) + ": residue code > 17");
            return CMGPU_EINVAL;
        }
    }
    return CMGPU_OK;
}

// Forward pieces (totscale, xC) and bias rows of every window, on the device
// (either output may be null).  The residue buffer is copied once.
int score_windows(const cmgpu_fwd_filter *f, cudaStream_t st, const uint8_t *dsq_all, int64_t dsq_len,
                  const cmgpu_window *wins, int32_t nwin, const uint8_t *want_fwd, std::vector<float> *fwd_ts,
                  std::vector<float> *fwd_xc, std::vector<float> *bias_rows) {
    cmgpu_fwd_filter *mf = const_cast<cmgpu_fwd_filter *>(f);
    mf->last_ms = 0;
    mf->last_cells = 0;
    mf->last_launches = 0;
    if (nwin == 0) return CMGPU_OK;
    const FwdHost &h = f->host;
    FWD_TRY(cudaSetDevice(f->device));
    // Forward windows longest first (the groups' work queue), bias in input order
    std::vector<int32_t> order;
    for (int32_t k = 0; k < nwin; k++)
        if (fwd_ts && (!want_fwd || want_fwd[k])) order.push_back(k);
    std::stable_sort(order.begin(), order.end(), [&](int32_t a, int32_t b) {
        return (wins[a].j0 - wins[a].i0) > (wins[b].j0 - wins[b].i0);
    });
    const int32_t nf = (int32_t)order.size();
    std::vector<cmx::dev::FwdWin> fw((size_t)nf + (bias_rows ? nwin : 0));
    for (int32_t q = 0; q < nf; q++) {
        const cmgpu_window &w = wins[order[q]];
        fw[q] = {w.dsq_offset + w.i0, std::max(0, w.j0 - w.i0 + 1), 0};
    }
    if (bias_rows)
        for (int32_t k = 0; k < nwin; k++) {
            const cmgpu_window &w = wins[k];
            fw[(size_t)nf + k] = {w.dsq_offset + w.i0, std::max(0, w.j0 - w.i0 + 1), 0};
        }
    uint8_t *d_dsq = nullptr;
    cmx::dev::FwdWin *d_w = nullptr;
    float2 *d_out = nullptr;
    float *d_rows = nullptr;
    int *d_next = nullptr;
    cudaError_t e = cudaSuccess;
    if ((e = mf->arena.get(0, &d_dsq, (size_t)dsq_len)) != cudaSuccess ||
        (e = mf->arena.get(1, &d_w, sizeof(cmx::dev::FwdWin) * fw.size())) != cudaSuccess ||
        (e = mf->arena.get(2, &d_out, sizeof(float2) * std::max(nf, 1))) != cudaSuccess ||
        (e = mf->arena.get(3, &d_rows, sizeof(float) * (size_t)nwin)) != cudaSuccess ||
        (e = mf->arena.get(4, &d_next, sizeof(int))) != cudaSuccess) {
        set_error(std::string("cmgpu_fwd: ") + cudaGetErrorString(e));
        return CMGPU_ENOMEM;
    }
    FWD_TRY(cudaMemcpyAsync(d_dsq, dsq_all, (size_t)dsq_len, cudaMemcpyHostToDevice, st));
    FWD_TRY(cudaMemcpyAsync(d_w, fw.data(), sizeof(cmx::dev::FwdWin) * fw.size(), cudaMemcpyHostToDevice, st));
    FWD_TRY(cudaMemsetAsync(d_next, 0, sizeof(int), st));
    // launch shape: as many groups of four as fit, tables in shared memory
    // when they leave room for at least 16 groups
    const int nq = h.nq;
    const int gstride = ((12 * nq + 31) & ~31) + 4;
    const size_t tab_words = ((size_t)nq * T_N * 4 + (size_t)KP * h.rq * 4 + 31) & ~(size_t)31;
    int optin = 0, sms = 148;
    FWD_TRY(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, f->device));
    FWD_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, f->device));
    const size_t room = (size_t)optin / 4;  // words
    const bool ts = tab_words + (size_t)16 * gstride <= room / 2;
    int threads = 256;
    auto smem_words = [&](int thr) { return (ts ? tab_words : 0) + (size_t)(thr / 4) * gstride; };
    while (threads > 32 && smem_words(threads) > room / 2) threads /= 2;
    if (smem_words(threads) > room) {
        set_error("cmgpu_fwd: model too long for the shared-memory rows");
        return CMGPU_ENOSPACE;
    }
    const size_t smem = smem_words(threads) * 4;
    cudaEvent_t ev0 = f->t0, ev1 = f->t1;
    FWD_TRY(cudaEventRecord(ev0, st));
    if (bias_rows) {
        // the bias null (one thread per window, a few CTAs) beside the Forward kernel
        cmx::dev::BiasParams bp;
        std::memcpy(bp.eo, h.eo, sizeof bp.eo);
        std::memcpy(bp.t1, h.t1, sizeof bp.t1);
        FWD_TRY(cudaEventRecord(f->fork, st));
        FWD_TRY(cudaStreamWaitEvent(f->side, f->fork, 0));
        cmx::dev::bias_kernel<<<(nwin + 127) / 128, 128, 0, f->side>>>(bp, d_dsq, d_w + nf, nwin, d_rows);
        FWD_TRY(cudaGetLastError());
        FWD_TRY(cudaEventRecord(f->join, f->side));
        mf->last_launches++;
    }
    const bool regs = nq <= 32 && f->kernel != CMGPU_FWD_KERNEL_SHARED;
    if (nf > 0 && regs) {
        // the segment of each lane fits in registers
        auto kern = cmx::dev::fwd_reg_kernel(nq, h.M >= 100, std::make_integer_sequence<int, 31>());
        const size_t rsmem = (size_t)(nq * T_N * 4 + KP * h.rq * 4) * sizeof(float);
        FWD_TRY(cmx::allow_max_dynamic_smem(kern));
        int per_sm = 0;
        FWD_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 128, rsmem));
        const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((nf + 31) / 32, (int64_t)sms * std::max(per_sm, 1)));
        kern<<<grid, 128, rsmem, st>>>(f->d_ptab, h.rq, d_dsq, d_w, nf, d_next, d_out);
        FWD_TRY(cudaGetLastError());
        mf->last_launches++;
    } else if (nf > 0) {
        auto kern = ts ? cmx::dev::fwd_kernel<true> : cmx::dev::fwd_kernel<false>;
        FWD_TRY(cmx::allow_max_dynamic_smem(kern));
        int per_sm = 0;
        FWD_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem));
        const int groups = threads / 4;
        const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((nf + groups - 1) / groups,
                                                                    (int64_t)sms * std::max(per_sm, 1)));
        kern<<<grid, threads, smem, st>>>(f->d_tab, h.M, nq, h.rq, gstride, d_dsq, d_w, nf, d_next, d_out);
        FWD_TRY(cudaGetLastError());
        mf->last_launches++;
    }
    if (bias_rows) FWD_TRY(cudaStreamWaitEvent(st, f->join, 0));
    FWD_TRY(cudaEventRecord(ev1, st));
    std::vector<float2> out((size_t)nf);
    if (nf > 0) FWD_TRY(cudaMemcpyAsync(out.data(), d_out, sizeof(float2) * nf, cudaMemcpyDeviceToHost, st));
    if (bias_rows) {
        bias_rows->resize(nwin);
        FWD_TRY(cudaMemcpyAsync(bias_rows->data(), d_rows, sizeof(float) * nwin, cudaMemcpyDeviceToHost, st));
    }
    FWD_TRY(cudaStreamSynchronize(st));
    float ms = 0;
    cudaEventElapsedTime(&ms, ev0, ev1);
    mf->last_ms = ms;
    if (fwd_ts) {
        fwd_ts->assign(nwin, 0.0f);
        fwd_xc->assign(nwin, 0.0f);
        for (int32_t q = 0; q < nf; q++) {
            (*fwd_ts)[order[q]] = out[q].x;
            (*fwd_xc)[order[q]] = out[q].y;
            mf->last_cells += (int64_t)fw[q].L * h.M;
        }
    }
    return CMGPU_OK;
}

// the scores from their device pieces, as the reference finishes them
float fwd_final(float totscale, float xc, int32_t L) {
    const float pmove = (2.0f + 1.0f) / ((float)L + 2.0f + 1.0f);
    return (float)((double)totscale + std::log((double)xc * (double)pmove));
}

float bias_final(float rows, int32_t L) {
    if (L == 0) return 0.0f;
    const float lf = (float)L;
    const float p1 = lf / (lf + 1.0f);
    return rows + lf * std::log(p1) + std::log(1.0f - p1);
}

}  // namespace

extern "C" int cmgpu_fwd_filter_build(const cmgpu_p7_profile *p, const float *compo, double ftau, double flambda,
                                      int device, cmgpu_fwd_filter **out) {
    if (!p || !out || !compo || p->M < 1 || !p->mat || !p->trans) return CMGPU_EINVAL;
    *out = nullptr;
    auto *f = new (std::nothrow) cmgpu_fwd_filter();
    if (!f) return CMGPU_ENOMEM;
    build_host(p, compo, f->host);
    f->host.ftau = ftau;
    f->host.flambda = flambda;
    f->device = device;
    if (device >= 0) {
        cudaError_t e = cudaSetDevice(device);
        const size_t bytes = f->host.stab.size() * sizeof(float);
        if (e == cudaSuccess) e = cudaMalloc(&f->d_tab, bytes);
        if (e == cudaSuccess) e = cudaMemcpy(f->d_tab, f->host.stab.data(), bytes, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMalloc(&f->d_ptab, bytes);
        if (e == cudaSuccess) e = cudaMemcpy(f->d_ptab, f->host.ptab.data(), bytes, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&f->side, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&f->fork, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&f->join, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreate(&f->t0);
        if (e == cudaSuccess) e = cudaEventCreate(&f->t1);
        if (e != cudaSuccess) {
            set_error(std::string("cmgpu_fwd_filter_build: ") + cudaGetErrorString(e));
            delete f;
            return CMGPU_EDEVICE;
        }
    }
    *out = f;
    return CMGPU_OK;
}

extern "C" void cmgpu_fwd_filter_free(cmgpu_fwd_filter *f) { delete f; }

extern "C" int cmgpu_fwd_filter_tables(const cmgpu_fwd_filter *f, float *rfv, float *tr, int32_t cap, int32_t *m_out,
                                       float *eo, float *t1) {
    if (!f || !m_out) return CMGPU_EINVAL;
    const FwdHost &h = f->host;
    *m_out = h.M;
    if (!rfv && !tr) return CMGPU_OK;
    if (cap < h.M + 1) {
        set_error("cmgpu_fwd_filter_tables: capacity below M + 1 rows");
        return CMGPU_EOVERFLOW;
    }
    if (rfv) std::memcpy(rfv, h.rfv.data(), h.rfv.size() * sizeof(float));
    if (tr) std::memcpy(tr, h.tr.data(), h.tr.size() * sizeof(float));
    if (eo) std::memcpy(eo, h.eo, sizeof h.eo);
    if (t1) std::memcpy(t1, h.t1, sizeof h.t1);
    return CMGPU_OK;
}

extern "C" int cmgpu_fwd_score_batch(const cmgpu_fwd_filter *f, void *stream, const uint8_t *dsq_all, int64_t dsq_len,
                                     const cmgpu_window *wins, int32_t nwin, float *fwd_scores, float *bias_scores) {
    if (!f || !dsq_all || nwin < 0 || (nwin > 0 && !wins) || (!fwd_scores && !bias_scores)) return CMGPU_EINVAL;
    if (!f->d_tab) {
        set_error("cmgpu_fwd_score_batch: filter was built without a device");
        return CMGPU_EINVAL;
    }
    int rc = check_windows("cmgpu_fwd_score_batch", dsq_all, dsq_len, wins, nwin);
    if (rc) return rc;
    std::vector<float> ts, xc, rows;
    rc = score_windows(f, (cudaStream_t)stream, dsq_all, dsq_len, wins, nwin, nullptr, fwd_scores ? &ts : nullptr,
                       fwd_scores ? &xc : nullptr, bias_scores ? &rows : nullptr);
    if (rc) return rc;
    for (int32_t k = 0; k < nwin; k++) {
        const int32_t L = std::max(0, wins[k].j0 - wins[k].i0 + 1);
        if (fwd_scores) fwd_scores[k] = fwd_final(ts[k], xc[k], L);
        if (bias_scores) bias_scores[k] = bias_final(rows[k], L);
    }
    return CMGPU_OK;
}

extern "C" int cmgpu_fwd_filter_set_kernel(cmgpu_fwd_filter *f, int kernel) {
    if (!f || kernel < CMGPU_FWD_KERNEL_AUTO || kernel > CMGPU_FWD_KERNEL_SHARED) return CMGPU_EINVAL;
    f->kernel = kernel;
    return CMGPU_OK;
}

extern "C" int cmgpu_fwd_filter_stats(const cmgpu_fwd_filter *f, double *kernel_ms, int64_t *cells,
                                      int32_t *launches) {
    if (!f) return CMGPU_EINVAL;
    if (kernel_ms) *kernel_ms = f->last_ms;
    if (cells) *cells = f->last_cells;
    if (launches) *launches = f->last_launches;
    return CMGPU_OK;
}

namespace {

// p7_bg_null_one (src/cm_pipeline.rs:1122-1125)
double null_one(int64_t L) {
    const double p1 = (double)L / ((double)L + 1.0);
    return (double)L * std::log(p1) + std::log(1.0 - p1);
}

// esl_exp_surv (src/cp9.rs:6531-6537)
double exp_surv(double x, double mu, double lambda) { return x < mu ? 1.0 : std::exp(-lambda * (x - mu)); }

// esl_gumbel_surv (src/cm_pipeline.rs:1852-1861)
double gumbel_surv(double x, double mu, double lambda) {
    const double y = lambda * (x - mu);
    const double ey = -std::exp(-y);
    return std::fabs(ey) < 5e-9 ? -ey : 1.0 - std::exp(ey);
}

}  // namespace

extern "C" int cmgpu_f3_filter(const cmgpu_fwd_filter *ff, const cmgpu_msv_filter *mf, const cmgpu_vit_filter *vf,
                               void *stream, const uint8_t *dsq_all, int64_t dsq_len, const cmgpu_window *chunks,
                               int32_t nchunk, const cmgpu_f3_config *cfg, cmgpu_f1_window *out, int32_t cap,
                               int32_t *n_out, cmgpu_f3_acct *acct) {
    if (!ff || !dsq_all || !cfg || !n_out || nchunk < 0 || (nchunk > 0 && !chunks) || cap < 0) return CMGPU_EINVAL;
    *n_out = 0;
    if (((cfg->do_msv || cfg->do_msvbias) && !mf) || (cfg->do_vit && !vf)) {
        set_error("cmgpu_f3_filter: a stage is on without its filter");
        return CMGPU_EINVAL;
    }
    if ((cfg->do_msv && cfg->cmw < 1) || (!cfg->do_msv && cfg->maxw < 1)) {
        set_error("cmgpu_f3_filter: cmw (with SSV windows) or maxw (tiled windows) must be positive");
        return CMGPU_EINVAL;
    }
    if (!ff->d_tab) {
        set_error("cmgpu_f3_filter: filter was built without a device");
        return CMGPU_EINVAL;
    }
    int rc = check_windows("cmgpu_f3_filter", dsq_all, dsq_len, chunks, nchunk);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    double dev_ms = 0;
    int32_t dev_launches = 0;
    // windows: SSV (F1) or deterministic 2*maxW tiles (src/cm_pipeline.rs:1890-1915)
    std::vector<cmgpu_f1_window> w1;
    if (cfg->do_msv) {
        rc = cmx::f1_msv_windows_vec(mf, st, dsq_all, dsq_len, chunks, nchunk, cfg->f1, cfg->cmw, w1);
        if (rc) return rc;
        double ms = 0;
        int32_t l = 0;
        cmgpu_msv_filter_stats(mf, &ms, nullptr, &l);
        dev_ms += ms;
        dev_launches += l;
    } else {
        for (int32_t c = 0; c < nchunk; c++) {
            const int64_t n = std::max(0, chunks[c].j0 - chunks[c].i0 + 1), mw = cfg->maxw;
            int64_t nw = 1;
            if (n > 2 * mw) {
                nw += (n - 2 * mw) / (mw + 1);
                if ((n - 2 * mw) % (mw + 1) > 0) nw++;
            }
            for (int64_t q = 0; q < nw; q++) {
                const int64_t ws = 1 + q * (mw + 1);
                w1.push_back({ws, std::min(ws + 2 * mw - 1, n), 0.0f, c});
            }
        }
    }
    const int32_t nw = (int32_t)w1.size();
    std::vector<cmgpu_window> bw(nw);
    std::vector<int32_t> wlen(nw);
    for (int32_t k = 0; k < nw; k++) {
        const cmgpu_window &c = chunks[w1[k].chunk];
        bw[k] = {c.dsq_offset, (int32_t)(c.i0 + w1[k].start - 1), (int32_t)(c.i0 + w1[k].end - 1)};
        wlen[k] = (int32_t)(w1[k].end - w1[k].start + 1);
    }
    const bool need_bias = cfg->do_msvbias || (cfg->do_vit && cfg->do_vitbias) || (cfg->do_fwd && cfg->do_fwdbias);
    const bool gated = cfg->do_msvbias || cfg->do_vit;
    std::vector<float> ts, xc, rows;
    std::vector<float> msv_sc(nw), vit_sc(nw);
    std::vector<uint8_t> msv_ok(nw, 0), vit_ok(nw, 0);
    auto add_fwd_stats = [&]() {
        dev_ms += ff->last_ms;
        dev_launches += ff->last_launches;
    };
    // F3 and F3b scores in one pass when no earlier stage gates the windows
    if (nw > 0 && (need_bias || (cfg->do_fwd && !gated))) {
        rc = score_windows(ff, st, dsq_all, dsq_len, bw.data(), nw, nullptr,
                           cfg->do_fwd && !gated ? &ts : nullptr, cfg->do_fwd && !gated ? &xc : nullptr,
                           need_bias ? &rows : nullptr);
        if (rc) return rc;
        add_fwd_stats();
    }
    if (cfg->do_msvbias && nw > 0) {
        rc = cmgpu_msv_score_batch(mf, stream, dsq_all, dsq_len, bw.data(), nw, wlen.data(), msv_sc.data(),
                                   msv_ok.data());
        if (rc) return rc;
        double ms = 0;
        int32_t l = 0;
        cmgpu_msv_filter_stats(mf, &ms, nullptr, &l);
        dev_ms += ms;
        dev_launches += l;
    }
    const double ln2 = std::log(2.0);
    std::vector<uint8_t> s_f1b(nw, 1), s_f2(nw, 1), s_f2b(nw, 1), s_f3(nw, 0), s_f3b(nw, 0), reach(nw, 1);
    std::vector<float> bias(nw, 0.0f);
    if (need_bias)
        for (int32_t k = 0; k < nw; k++) bias[k] = bias_final(rows[k], wlen[k]);
    // F1b (src/cm_pipeline.rs:1963-1977)
    if (cfg->do_msvbias)
        for (int32_t k = 0; k < nw; k++)
            if (msv_ok[k] &&
                gumbel_surv(((double)msv_sc[k] - (double)bias[k]) / ln2, cfg->lmmu, cfg->lmlambda) > cfg->f1b) {
                s_f1b[k] = 0;
                reach[k] = 0;
            }
    // F2 / F2b (:1983-2016) on the F1b survivors
    if (cfg->do_vit) {
        std::vector<int32_t> idx;
        std::vector<cmgpu_window> sub;
        for (int32_t k = 0; k < nw; k++)
            if (reach[k]) {
                idx.push_back(k);
                sub.push_back(bw[k]);
            }
        std::vector<float> sc(sub.size());
        std::vector<uint8_t> ok(sub.size());
        if (!sub.empty()) {
            rc = cmgpu_vit_score_batch(vf, stream, dsq_all, dsq_len, sub.data(), (int32_t)sub.size(), sc.data(),
                                       ok.data());
            if (rc) return rc;
            double ms = 0;
            int32_t l = 0;
            cmgpu_vit_filter_stats(vf, &ms, nullptr, &l);
            dev_ms += ms;
            dev_launches += l;
        }
        for (size_t q = 0; q < idx.size(); q++) {
            const int32_t k = idx[q];
            if (!ok[q]) continue;  // 16-bit overflow: a very high score, survives
            const double nullsc = null_one(wlen[k]);
            if (gumbel_surv(((double)sc[q] - nullsc) / ln2, cfg->lvmu, cfg->lvlambda) > cfg->f2) {
                s_f2[k] = s_f2b[k] = 0;
                reach[k] = 0;
                continue;
            }
            if (cfg->do_vitbias &&
                gumbel_surv(((double)sc[q] - (double)bias[k]) / ln2, cfg->lvmu, cfg->lvlambda) > cfg->f2b) {
                s_f2b[k] = 0;
                reach[k] = 0;
            }
        }
    }
    // F3 Forward on the windows that reach it, when earlier stages gated them
    if (cfg->do_fwd && gated && nw > 0) {
        rc = score_windows(ff, st, dsq_all, dsq_len, bw.data(), nw, reach.data(), &ts, &xc, nullptr);
        if (rc) return rc;
        add_fwd_stats();
    }
    std::vector<float> wb(nw, -999.0f);
    for (int32_t k = 0; k < nw; k++) {
        if (!reach[k]) continue;
        float fwdsc = 0.0f;
        if (cfg->do_fwd) {
            fwdsc = fwd_final(ts[k], xc[k], wlen[k]);
            const double wsc = ((double)fwdsc - null_one(wlen[k])) / ln2;
            wb[k] = (float)wsc;
            if (exp_surv(wsc, ff->host.ftau, ff->host.flambda) > cfg->f3) continue;
        }
        s_f3[k] = 1;
        if (cfg->do_fwd && cfg->do_fwdbias) {
            const double wsc = ((double)fwdsc - (double)bias[k]) / ln2;
            wb[k] = (float)wsc;
            if (exp_surv(wsc, ff->host.ftau, ff->host.flambda) > cfg->f3b) continue;
        }
        s_f3b[k] = 1;
    }
    // per chunk: merge the survivors that overlap or abut (:2056-2103) and
    // count the residues past each stage (:2105-2164)
    cmgpu_f3_acct a{};
    std::vector<cmgpu_f1_window> res;
    for (int32_t k0 = 0; k0 < nw;) {
        int32_t k1 = k0;
        while (k1 < nw && w1[k1].chunk == w1[k0].chunk) k1++;
        std::vector<cmgpu_f1_window> sv;
        for (int32_t k = k0; k < k1; k++)
            if (s_f3b[k]) sv.push_back({w1[k].start, w1[k].end, wb[k], w1[k].chunk});
        for (size_t i = 0; i < sv.size();) {
            size_t i2 = i + 1;
            cmgpu_f1_window m = sv[i];
            while (i2 < sv.size() && m.end + 1 >= sv[i2].start) {
                m.end = sv[i2].end;
                m.score = std::max(m.score, sv[i2].score);
                i2++;
            }
            res.push_back(m);
            i = i2;
        }
        int64_t *np[5] = {&a.n_past_msvbias, &a.n_past_vit, &a.n_past_vitbias, &a.n_past_fwd, &a.n_past_fwdbias};
        int64_t *pp[5] = {&a.pos_past_msvbias, &a.pos_past_vit, &a.pos_past_vitbias, &a.pos_past_fwd,
                          &a.pos_past_fwdbias};
        const std::vector<uint8_t> *sf[5] = {&s_f1b, &s_f2, &s_f2b, &s_f3, &s_f3b};
        a.n_past_msv += k1 - k0;
        for (int32_t k = k0; k < k1; k++) {
            a.pos_past_msv += wlen[k];
            for (int s = 0; s < 5; s++)
                if ((*sf[s])[k]) {
                    (*np[s])++;
                    *pp[s] += wlen[k];
                }
            if (k > k0) {
                const int64_t ov = w1[k - 1].end - w1[k].start + 1;
                if (ov > 0) {
                    a.pos_past_msv -= ov;
                    for (int s = 0; s < 5; s++)
                        if ((*sf[s])[k] && (*sf[s])[k - 1]) *pp[s] -= ov;
                }
            }
        }
        k0 = k1;
    }
    cmgpu_fwd_filter *mff = const_cast<cmgpu_fwd_filter *>(ff);
    mff->last_ms = dev_ms;
    mff->last_launches = dev_launches;
    if (acct) *acct = a;
    *n_out = (int32_t)res.size();
    if ((int64_t)res.size() > cap) {
        set_error("cmgpu_f3_filter: output capacity too small");
        return CMGPU_EOVERFLOW;
    }
    if (out) std::copy(res.begin(), res.end(), out);
    return CMGPU_OK;
}
