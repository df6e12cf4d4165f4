// C ABI of libcmscan_gpu.so (include/cmscan_gpu.h): model upload, workspaces,
// batching of windows into work items, the scan launch, and the host-side
// hit reporting.
//
// The device returns every reportable cell: (j, d) with bestsc >= cutoff.
// The host then replays, per window and column, the reference's greedy
// report (report_hits_greedily, src/cm_nohmm.rs:769-812) with the null3
// correction in double precision (score_correction_null3, src/cp9.rs:6516)
// and the greedy overlap removal (src/cp9.rs:6544-6574).  null3 can only
// lower a score, so the cells the device returns are a superset of what the
// reference could report, and the replay sees them in the reference's order
// (j ascending, d ascending).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/cmscan_gpu.h"
#include "cm_internal.h"
#include "model_internal.h"
#include "qdb_kernel.h"
#include "qdb_plan.h"
#include "sweep_kernel.h"

namespace cmx {

static thread_local std::string g_err;
void set_error(const std::string &msg) { g_err = msg; }

bool build_plan(const cmgpu_cm *cm, int semiring, int qdbidx, Plan &p);
void count_column_public(const cmgpu_cm *cm, const Plan &p, int qdbidx, int jrow, double &cells, double &terms);

#define CUDA_TRY(call)                                                                          \
    do {                                                                                        \
        cudaError_t e_ = (call);                                                                \
        if (e_ != cudaSuccess) {                                                                \
            set_error(std::string(#call) + ": " + cudaGetErrorString(e_));                      \
            return CMGPU_EDEVICE;                                                               \
        }                                                                                       \
    } while (0)

template <class T>
static int upload_vec(T **dst, const std::vector<T> &v) {
    size_t n = std::max<size_t>(v.size(), 1);
    CUDA_TRY(cudaMalloc((void **)dst, n * sizeof(T)));
    if (!v.empty()) CUDA_TRY(cudaMemcpy(*dst, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
    return CMGPU_OK;
}

}  // namespace cmx

using namespace cmx;

struct cmgpu_workspace {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // device buffers (grow only)
    uint8_t *d_dsq = nullptr;
    size_t dsq_cap = 0;
    WorkItem *d_items = nullptr;
    size_t items_cap = 0;
    Cand *d_cands = nullptr;
    size_t cands_cap = 0;
    int *d_counters = nullptr;  // [0] next item, [1] candidate count
    uint32_t *d_deck = nullptr;
    size_t deck_cap = 0;  // elements
    uint32_t *d_sweep = nullptr;  // node-sweep kernel: per-warp decks and BEGL rings
    size_t sweep_cap = 0;         // elements
    // host staging
    Cand *h_cands = nullptr;
    size_t h_cands_cap = 0;
    int *h_counters = nullptr;
    // launch shape
    int threads = 512;
    int ctas_per_sm = 0;  // 0 = tuned
    int chunk = 0;        // 0 = auto
    int lanes = 0;        // 0 = tuned
    int kernel = 0;       // CMGPU_KERNEL_*
    int sm_count = 148;
    cmgpu_stats stats{};
    ~cmgpu_workspace() {
        cudaFree(d_dsq);
        cudaFree(d_items);
        cudaFree(d_cands);
        cudaFree(d_counters);
        cudaFree(d_deck);
        cudaFree(d_sweep);
        cudaFreeHost(h_cands);
        cudaFreeHost(h_counters);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (own_stream && stream) cudaStreamDestroy(stream);
    }
};

namespace cmx {

static int get_plan(cmgpu_model *m, int semiring, int qdbidx, DevPlan **out) {
    std::lock_guard<std::mutex> lk(m->mu);
    int key = semiring * 8 + qdbidx;
    auto it = m->plans.find(key);
    if (it != m->plans.end()) {
        *out = it->second.get();
        return CMGPU_OK;
    }
    std::unique_ptr<DevPlan> dp(new DevPlan());
    if (!build_plan(&m->cm.view, semiring, qdbidx, dp->host)) return CMGPU_EINVAL;
    const Plan &p = dp->host;
    CUDA_TRY(cudaSetDevice(m->device));
    int rc;
    if ((rc = upload_vec(&dp->states, p.states))) return rc;
    if ((rc = upload_vec(&dp->chunks, p.chunks))) return rc;
    if ((rc = upload_vec(&dp->begins, p.begins))) return rc;
    if ((rc = upload_vec(&dp->level_start, p.level_start))) return rc;
    if ((rc = upload_vec(&dp->wb, p.wb))) return rc;
    if ((rc = upload_vec(&dp->cb, p.cb))) return rc;
    if ((rc = upload_vec(&dp->init_off, p.init_off))) return rc;
    if ((rc = upload_vec(&dp->init_val, p.init_val))) return rc;
    if ((rc = upload_vec(&dp->tsc, p.tsc))) return rc;
    if ((rc = upload_vec(&dp->endsc, p.endsc))) return rc;
    if ((rc = upload_vec(&dp->beginsc, p.beginsc))) return rc;
    if ((rc = upload_vec(&dp->beginsc_all, p.beginsc_all))) return rc;
    if ((rc = upload_vec(&dp->esc, p.esc))) return rc;
    if ((rc = upload_vec(&dp->el_sca, p.el_sca))) return rc;
    if ((rc = upload_vec(&dp->esc_c, p.esc_c))) return rc;
    // node-sweep plan
    {
        std::string why;
        dp->sw_ok = build_sweep_plan(&m->cm.view, p, qdbidx, dp->sw, &why);
        dp->sw_why = why;
        if ((rc = upload_vec(&dp->init0, p.init0))) return rc;
        if (dp->sw_ok) {
            std::vector<uint8_t> kid = dp->sw.kid;
            kid.resize((kid.size() + 3) & ~(size_t)3, 0);
            if ((rc = upload_vec(&dp->sw_st, dp->sw.st))) return rc;
            if ((rc = upload_vec(&dp->sw_kid, kid))) return rc;
            if ((rc = upload_vec(&dp->sw_nodes, dp->sw.nodes))) return rc;
            if ((rc = upload_vec(&dp->sw_io, dp->sw.io))) return rc;
            if ((rc = upload_vec(&dp->sw_bifs, dp->sw.bifs))) return rc;
        }
    }
    // per-column work counts by row limit
    const int W = p.W;
    dp->cells_prefix.assign(W + 1, 0.0);
    dp->terms_prefix.assign(W + 1, 0.0);
    for (int jr = 1; jr <= W; jr++) {
        double c = 0, t = 0;
        count_column_public(&m->cm.view, p, qdbidx, jr, c, t);
        dp->cells_prefix[jr] = dp->cells_prefix[jr - 1] + c;
        dp->terms_prefix[jr] = dp->terms_prefix[jr - 1] + t;
        if (jr == W) {
            dp->cells_full = c;
            dp->terms_full = t;
        }
    }
    *out = dp.get();
    m->plans[key] = std::move(dp);
    return CMGPU_OK;
}

// exact reference cells/terms of a window of length L
static void window_work(const DevPlan *dp, int64_t L, double &cells, double &terms) {
    const int W = dp->host.W;
    int64_t warm = std::min<int64_t>(L, W - 1);
    cells = dp->cells_prefix[warm];
    terms = dp->terms_prefix[warm];
    if (L > warm) {
        cells += dp->cells_full * (double)(L - warm);
        terms += dp->terms_full * (double)(L - warm);
    }
}

template <class T>
static int ensure_dev(T **p, size_t *cap, size_t n) {
    if (n <= *cap && *p) return CMGPU_OK;
    size_t nc = std::max<size_t>(n, *cap * 3 / 2 + 16);
    cudaFree(*p);
    *p = nullptr;
    *cap = 0;
    CUDA_TRY(cudaMalloc((void **)p, nc * sizeof(T)));
    *cap = nc;
    return CMGPU_OK;
}

static int ensure_host_cands(cmgpu_workspace *ws, size_t n) {
    if (n <= ws->h_cands_cap && ws->h_cands) return CMGPU_OK;
    size_t nc = std::max<size_t>(n, ws->h_cands_cap * 3 / 2 + 16);
    cudaFreeHost(ws->h_cands);
    ws->h_cands = nullptr;
    ws->h_cands_cap = 0;
    CUDA_TRY(cudaMallocHost((void **)&ws->h_cands, nc * sizeof(Cand)));
    ws->h_cands_cap = nc;
    return CMGPU_OK;
}

// ---------------------------------------------------------------------------
// host-side reporting
// ---------------------------------------------------------------------------
static inline double sre_log2d(double x) { return x > 0.0 ? std::log(x) * 1.44269504 : -1.0e36; }

static float flogsum_host(const std::vector<float> &tbl, float s1, float s2) {
    float mx = std::max(s1, s2), mn = std::min(s1, s2);
    if (mn == -INFINITY || (mx - mn) >= 23.0f) return mx;
    return mx + tbl[(size_t)((mx - mn) * 1000.0f)];
}

// score_correction_null3 (src/cp9.rs:6516-6528)
static float null3_correction(const cmgpu_model *m, const float *comp, int len) {
    float score = 0.0f;
    for (int a = 0; a < 4; a++) {
        double term = sre_log2d((double)(comp[a] / m->cm.view.null[a])) * (double)comp[a] * (double)len;
        score = (float)((double)score + term);
    }
    score = (float)((double)score + sre_log2d((double)m->cm.view.n3_omega));
    return flogsum_host(m->flog, 0.0f, score);
}

float null3_corr(const cmgpu_model *m, const float *comp, int len) { return null3_correction(m, comp, len); }

static inline float raw_bits(int semiring, uint32_t raw) {
    if (semiring == CMGPU_INSIDE_I32) {
        int32_t s = (int32_t)raw;
        return s == -INFTY ? IMPOSSIBLE : (float)((double)s / INTSCALE);
    }
    float f;
    std::memcpy(&f, &raw, 4);
    return f;
}

// remove_overlaps_greedy (src/cp9.rs:6544-6574): hits sorted by score
// (descending, stable) then start; a hit is removed when it overlaps an
// earlier hit that was kept.  The kept hits are disjoint, so they are held
// in a map ordered by start: the only kept hit that can overlap [i, j] is the
// one with the largest start <= j, and it overlaps when its end >= i.  Same
// result as the pairwise scan, in O(n log n).
static void remove_overlaps(std::vector<cmgpu_hit> &h) {
    std::stable_sort(h.begin(), h.end(), [](const cmgpu_hit &a, const cmgpu_hit &b) {
        if (a.score != b.score) return a.score > b.score;
        return a.i < b.i;
    });
    std::map<int32_t, int32_t> kept;  // start -> end
    size_t o = 0;
    for (size_t x = 0; x < h.size(); x++) {
        auto it = kept.upper_bound(h[x].j);
        if (it != kept.begin() && std::prev(it)->second >= h[x].i) continue;
        kept.emplace(h[x].i, h[x].j);
        h[o++] = h[x];
    }
    h.resize(o);
}

// Replays report_hits_greedily for one window from its candidate cells
// (sorted by j, d).  frame = window frame (host), needed for null3.
void report_window(const cmgpu_model *m, int semiring, const Cand *c, size_t n, const uint8_t *frame,
                          int32_t i0, float cutoff, int do_null3, std::vector<cmgpu_hit> &out) {
    std::vector<cmgpu_hit> tmp;
    // prefix counts of canonical residues over the candidates' span
    std::vector<int32_t> pre;
    int32_t lo = 0;
    if (do_null3 && n) {
        int32_t mini = c[0].j, maxj = c[0].j;
        for (size_t k = 0; k < n; k++) {
            mini = std::min(mini, c[k].j - c[k].d + 1);
            maxj = std::max(maxj, c[k].j);
        }
        lo = std::max(i0, mini) - 1;
        pre.assign((size_t)(maxj - lo + 1) * 4, 0);
        for (int32_t p = lo + 1; p <= maxj; p++) {
            for (int a = 0; a < 4; a++) pre[(size_t)(p - lo) * 4 + a] = pre[(size_t)(p - 1 - lo) * 4 + a];
            uint8_t r = frame[p];
            if (r < 4) pre[(size_t)(p - lo) * 4 + r]++;
        }
    }
    size_t k = 0;
    while (k < n) {
        int32_t j = c[k].j;
        float max_reported = IMPOSSIBLE;
        for (; k < n && c[k].j == j; k++) {
            int32_t d = c[k].d, i = j - d + 1;
            float hit_sc = raw_bits(semiring, c[k].raw);
            float bias = 0.0f;
            if (!(hit_sc > max_reported && hit_sc >= cutoff && hit_sc > IMPOSSIBLE + 1.0f)) continue;
            bool do_report = true;
            if (do_null3) {
                float comp[4];
                for (int a = 0; a < 4; a++) {
                    int32_t cnt = pre[(size_t)(j - lo) * 4 + a] - pre[(size_t)(i - 1 - lo) * 4 + a];
                    comp[a] = (float)(double)cnt;
                }
                float sum = 0.0f;
                for (int a = 0; a < 4; a++) sum += comp[a];
                if (sum > 0.0f)
                    for (int a = 0; a < 4; a++) comp[a] /= sum;
                else
                    for (int a = 0; a < 4; a++) comp[a] = 1.0f / 4.0f;
                float corr = null3_correction(m, comp, d);
                hit_sc -= corr;
                bias = corr;
                do_report = hit_sc > max_reported && hit_sc >= cutoff;
            }
            if (do_report) {
                tmp.push_back(cmgpu_hit{i, j, hit_sc, bias});
                max_reported = hit_sc;
            }
        }
    }
    remove_overlaps(tmp);
    out.insert(out.end(), tmp.begin(), tmp.end());
}

// ---------------------------------------------------------------------------
// the batched scan
// ---------------------------------------------------------------------------
struct WinDesc {
    int64_t off;
    int32_t i0, j0;
};

static int run_scan(cmgpu_model *m, cmgpu_workspace *ws, int semiring, int qdbidx, const uint8_t *d_dsq,
                    const uint8_t *h_dsq, int64_t dsq_len, const std::vector<WinDesc> &wins, float cutoff,
                    int do_null3, bool plain, std::vector<std::vector<cmgpu_hit>> &hits_per_win,
                    std::vector<Cand> *cells_out = nullptr, bool calib = false) {
    if (semiring != CMGPU_CYK_F32 && semiring != CMGPU_INSIDE_I32) {
        set_error("unknown semiring");
        return CMGPU_EINVAL;
    }
    if (qdbidx < 0 || qdbidx > 2) {
        set_error("unknown band set");
        return CMGPU_EINVAL;
    }
    DevPlan *dp = nullptr;
    int rc = get_plan(m, semiring, qdbidx, &dp);
    if (rc) return rc;
    const Plan &pl = dp->host;
    CUDA_TRY(cudaSetDevice(ws->device));
    hits_per_win.assign(wins.size(), {});
    memset(&ws->stats, 0, sizeof(ws->stats));

    ScanParams sp{};
    sp.states = dp->states;
    sp.wb = dp->wb;
    sp.cb = dp->cb;
    sp.chunks = dp->chunks;
    sp.level_start = dp->level_start;
    sp.nlev = (int)pl.level_start.size() - 1;
    sp.nchunks = (int)pl.chunks.size();
    sp.tsc = dp->tsc;
    sp.endsc = dp->endsc;
    sp.esc = dp->esc;
    sp.el_sca = dp->el_sca;
    sp.esc_c = dp->esc_c;
    sp.n_esc_c = (int)pl.esc_c.size();
    sp.begins = dp->begins;
    sp.beginsc = dp->beginsc;
    sp.nbegin = (int)pl.begins.size();
    sp.init_off = dp->init_off;
    sp.init_val = dp->init_val;
    sp.ninit = (int)pl.init_off.size();
    sp.M = pl.M;
    sp.W = pl.W;
    sp.root_dn = pl.root_dn;
    sp.root_dxcap = pl.root_dxcap;
    sp.root_cnum = pl.root_cnum;
    sp.local = pl.local ? 1 : 0;
    sp.inside = semiring == CMGPU_INSIDE_I32;
    // integer Inside with local begins: begin states post their cells to a
    // per-lane ROOT row (an atomic max) instead of ROOT scanning every begin
    // state per cell; only when the rows are small and no insert state is a
    // begin state (inserts are relaxed outside the chunk path)
    {
        bool ok = sp.inside && sp.local && (size_t)MAX_LANES * (pl.root_dxcap + 1) * 4 <= 64 * 1024;
        for (size_t v = 0; ok && v < pl.states.size(); v++)
            if ((pl.states[v].flags & SF_BEGIN) && (pl.states[v].type == IL_ST || pl.states[v].type == IR_ST))
                ok = false;
        sp.fuse_begin = ok ? 1 : 0;
        sp.beginsc_all = dp->beginsc_all;
    }
    sp.deck_elems = pl.deck_elems;
    // cmcalibrate's scan: bit-score order of the local begins, and the
    // report pre-filter (its cutoff of -inf makes every ROOT cell reportable)
    sp.begin_key = calib ? 1 : 0;
    sp.prefilter = calib ? 1 : 0;
    sp.do_null3 = do_null3 ? 1 : 0;
    for (int a = 0; a < 4; a++) sp.pf_null[a] = m->cm.view.null[a];
    sp.pf_omega = m->cm.view.n3_omega;
    // per-state tables in global memory when they alone would fill most of
    // the shared memory (models of a few thousand states)
    sp.tables_global = 0;
    if ((size_t)scan_layout(sp, 1, false).words * 4 > 120 * 1024) sp.tables_global = 1;
    sp.ilog = m->ilog;
    sp.ilog_nz = m->ilog_nz;
    sp.dsq = d_dsq;
    sp.cutoff = cutoff;

    // kernel choice
    if (calib && ws->kernel == CMGPU_KERNEL_SWEEP) {
        set_error("cmcalibrate's scan runs on the level kernel only");
        return CMGPU_EINVAL;
    }
    if (ws->kernel == CMGPU_KERNEL_SWEEP && !dp->sw_ok) {
        set_error("node-sweep kernel does not apply to this model: " + dp->sw_why);
        return CMGPU_EINVAL;
    }
    // AUTO takes the level kernel: measured faster on every workload here
    const bool sweep = dp->sw_ok && ws->kernel == CMGPU_KERNEL_SWEEP;
    const size_t SMEM_CAP = 227 * 1024 - 1024, SM_CAP = 228 * 1024;
    const int threads = ws->threads;
    int best_c = 0, best_l = 0;
    bool deck_smem = false;
    SweepParams swp{};
    if (sweep) {
        // one CTA per SM with as many warps (one work item each) as fit
        const SweepPlan &sw = dp->sw;
        swp.st = dp->sw_st;
        swp.kid = dp->sw_kid;
        swp.nodes = dp->sw_nodes;
        swp.io = dp->sw_io;
        swp.bifs = dp->sw_bifs;
        swp.tsc = dp->tsc;
        swp.endsc = dp->endsc;
        swp.init0 = dp->init0;
        swp.bsv = dp->beginsc_all;
        swp.esc = dp->esc;
        swp.esc_c = dp->esc_c;
        swp.el_sca = dp->el_sca;
        swp.ilog = m->ilog;
        swp.ilog_nz = m->ilog_nz;
        swp.M = pl.M;
        swp.W = pl.W;
        swp.S = sw.S;
        swp.RW = sw.RW;
        swp.nnodes = (int)sw.nodes.size();
        swp.nio = (int)sw.io.size();
        swp.nbif = (int)sw.bifs.size();
        swp.n_esc_c = (int)pl.esc_c.size();
        swp.local = pl.local ? 1 : 0;
        swp.inside = sp.inside;
        swp.dsq = d_dsq;
        swp.cutoff = cutoff;
        swp.deck_words = sw.deck_words;
        swp.gstride = ((sw.deck_words + sw.ring_words) + 63) & ~(int64_t)63;
        const int wmax = ws->lanes > 0 ? std::min(ws->lanes, SW_MAX_WARPS) : SW_MAX_WARPS;
        for (int w = wmax; w >= 1; w--) {
            swp.warps = w;
            swp.lay = sweep_layout(swp, w);
            if ((size_t)swp.lay.words * 4 > SMEM_CAP) continue;
            if (sweep_occupancy(swp, w * 32) < 1) continue;
            best_l = w;
            break;
        }
        if (best_l < 1) {
            set_error("node-sweep kernel: the model tables leave no room for a warp in shared memory");
            return CMGPU_EDEVICE;
        }
        swp.warps = best_l;
        swp.lay = sweep_layout(swp, best_l);
        best_c = 1;
    } else {
        // launch shape: lanes (work items per CTA) x CTAs per SM.  Decks go to
        // shared memory when at least 3 lanes fit per SM; otherwise to global
        // memory (L2-resident) with 8 lanes per CTA, which keeps more
        // independent work in flight per SM.
        auto occ_for = [&](int l, bool smem_deck) {
            sp.lanes = l;
            sp.deck_smem = smem_deck ? 1 : 0;
            sp.lay = scan_layout(sp, l, smem_deck);
            return scan_occupancy(sp, threads);
        };
        for (int c = 1; c <= 4; c++) {
            if (ws->ctas_per_sm > 0 && c != ws->ctas_per_sm) continue;
            size_t cap = std::min(SMEM_CAP, SM_CAP / c - 1024);
            for (int t = MAX_LANES; t >= 1; t--) {
                if (ws->lanes > 0 && t != ws->lanes) continue;
                if ((size_t)scan_layout(sp, t, true).words * 4 > cap) continue;
                if (occ_for(t, true) >= c && c * t > best_c * best_l) {
                    best_c = c;
                    best_l = t;
                }
                break;
            }
        }
        bool forced = ws->lanes > 0 || ws->ctas_per_sm > 0;
        if (best_c * best_l < 3 && !(forced && best_c > 0)) best_c = 0;
        if (best_c > 0) {
            deck_smem = true;
        } else {
            best_l = ws->lanes > 0 ? ws->lanes : MAX_LANES;
            best_c = ws->ctas_per_sm > 0 ? ws->ctas_per_sm : 1;
        }
        int occ = occ_for(best_l, deck_smem);
        if (occ < 1) {
            set_error("scan kernel cannot be resident with this shape");
            return CMGPU_EDEVICE;
        }
        best_c = std::min(best_c, occ);
    }
    const int max_ctas = ws->sm_count * best_c;

    // work items: pieces of `chunk` reported columns plus W-1 warm-up columns.
    // The batch shares one cost-ordered queue; the plain comparator launches
    // once per window over that window's own pieces.
    std::vector<WorkItem> items;
    std::vector<size_t> win_first;  // plain: first item of each window
    int64_t total_cols = 0;
    for (auto &w : wins) total_cols += std::max<int64_t>(0, (int64_t)w.j0 - w.i0 + 1);
    const int W = pl.W;
    // Small batches -- too few columns to give every lane slot one piece of
    // 2W -- are latency bound: a lane scans its item's columns one after
    // another, and a CTA's time per column grows with its lanes.  Such a
    // batch is cut into about one piece per CTA, and each CTA takes only the
    // few lanes the pieces need (below).
    const bool small_batch = !sweep && !deck_smem && !plain && ws->chunk <= 0 && ws->lanes <= 0 &&
                             total_cols < (int64_t)max_ctas * best_l * 2 * W;
    auto chunk_for = [&](int64_t cols) -> int64_t {
        int64_t chunk = ws->chunk;
        if (chunk <= 0 && small_batch) {
            chunk = (cols + max_ctas - 1) / max_ctas;
            chunk = std::max<int64_t>(chunk, 2 * (int64_t)W);
            chunk = std::min<int64_t>(chunk, 32768);
        } else if (chunk <= 0) {
            // about four items per lane slot, but no piece shorter than 2W (the
            // W-1 warm-up columns are overhead) and none longer than 32768
            chunk = cols / std::max<int64_t>(1, (int64_t)max_ctas * best_l * 4);
            chunk = std::max<int64_t>(chunk, 2 * (int64_t)W);
            chunk = std::min<int64_t>(chunk, 32768);
        }
        return chunk;
    };
    const int64_t batch_chunk = chunk_for(total_cols);
    for (size_t wi = 0; wi < wins.size(); wi++) {
        const WinDesc &w = wins[wi];
        win_first.push_back(items.size());
        if (w.j0 < w.i0) continue;
        double c = 0, t = 0;
        window_work(dp, (int64_t)w.j0 - w.i0 + 1, c, t);
        ws->stats.cells += c;
        ws->stats.terms += t;
        ws->stats.residues += (double)w.j0 - w.i0 + 1;
        const int64_t chunk = plain ? chunk_for((int64_t)w.j0 - w.i0 + 1) : batch_chunk;
        for (int64_t r0 = w.i0; r0 <= w.j0; r0 += chunk) {
            int64_t r1 = std::min<int64_t>(w.j0, r0 + chunk - 1);
            int64_t js = std::max<int64_t>(w.i0, r0 - (W - 1));
            items.push_back(WorkItem{w.off, (int32_t)js, (int32_t)r1, (int32_t)r0, (int32_t)wi});
        }
    }
    win_first.push_back(items.size());
    if (!plain)
        std::stable_sort(items.begin(), items.end(), [](const WorkItem &a, const WorkItem &b) {
            return (a.jend - a.jstart) > (b.jend - b.jstart);
        });
    ws->stats.work_items = (int64_t)items.size();
    ws->stats.deck_in_smem = deck_smem ? 1 : 0;
    ws->stats.lanes = best_l;
    ws->stats.kernel = sweep ? CMGPU_KERNEL_SWEEP : CMGPU_KERNEL_LEVEL;
    if (items.empty()) return CMGPU_OK;

    if ((rc = ensure_dev(&ws->d_items, &ws->items_cap, items.size()))) return rc;
    CUDA_TRY(cudaMemcpyAsync(ws->d_items, items.data(), items.size() * sizeof(WorkItem), cudaMemcpyHostToDevice,
                             ws->stream));
    // Room for one reportable cell per four columns (4 bytes of device memory
    // per residue): batches with homologs in a tenth of their sequences stay
    // well inside it, so the scan is not repeated with a larger buffer.
    const size_t cand_cap = std::max<size_t>({ws->cands_cap, (size_t)1 << 16, (size_t)(total_cols / 4)});
    if ((rc = ensure_dev(&ws->d_cands, &ws->cands_cap, cand_cap))) return rc;
    if (!sweep && !deck_smem && (int64_t)items.size() < best_l) {
        // fewer work items than lanes: no deck for lanes that would stay idle
        best_l = (int)items.size();
        sp.lanes = best_l;
        sp.lay = scan_layout(sp, best_l, false);
        ws->stats.lanes = best_l;
    } else if (small_batch) {
        // a small batch: spread its pieces over every SM, a few lanes each
        const int l = (int)std::min<int64_t>(best_l, ((int64_t)items.size() + max_ctas - 1) / max_ctas);
        if (l < best_l) {
            best_l = std::max(1, l);
            sp.lanes = best_l;
            sp.lay = scan_layout(sp, best_l, false);
            ws->stats.lanes = best_l;
        }
    }
    int ctas = (int)std::min<int64_t>(((int64_t)items.size() + best_l - 1) / best_l, max_ctas);
    if (!sweep && !deck_smem) {
        // global decks of large models: keep them within half of the free device memory
        size_t freeb = 0, totalb = 0;
        CUDA_TRY(cudaMemGetInfo(&freeb, &totalb));
        const size_t per_cta = (((size_t)pl.deck_elems + 31) & ~(size_t)31) * 4 * (size_t)best_l;
        const size_t have = freeb / 2 + (ws->deck_cap * 4);
        const int fit = (int)std::max<size_t>(1, have / std::max<size_t>(per_cta, 1));
        ctas = std::min(ctas, fit);
    }
    ws->stats.ctas = ctas;
    if (sweep) {
        if ((rc = ensure_dev(&ws->d_sweep, &ws->sweep_cap, (size_t)swp.gstride * (size_t)ctas * (size_t)best_l)))
            return rc;
        swp.gmem = ws->d_sweep;
        swp.next_item = ws->d_counters;
        swp.cand_count = ws->d_counters + 1;
    } else if (!deck_smem) {
        size_t stride = ((size_t)pl.deck_elems + 31) & ~(size_t)31;
        if ((rc = ensure_dev(&ws->d_deck, &ws->deck_cap, stride * (size_t)ctas * (size_t)best_l))) return rc;
        sp.deck_global = ws->d_deck;
        sp.deck_stride = (int64_t)stride;
    }
    sp.next_item = ws->d_counters;
    sp.cand_count = ws->d_counters + 1;

    // one launch over items [first, first + n) on `grid` CTAs
    auto launch = [&](size_t first, size_t n, int grid) -> cudaError_t {
        if (sweep) {
            swp.items = ws->d_items + first;
            swp.nitems = (int)n;
            swp.item_base = (int)first;
            swp.cands = ws->d_cands;
            swp.cand_cap = (int)std::min<size_t>(ws->cands_cap, (size_t)INT32_MAX);
            return sweep_launch(swp, grid, ws->stream);
        }
        sp.items = ws->d_items + first;
        sp.nitems = (int)n;
        sp.item_base = (int)first;
        sp.cands = ws->d_cands;
        sp.cand_cap = (int)std::min<size_t>(ws->cands_cap, (size_t)INT32_MAX);
        return scan_launch(sp, grid, threads, ws->stream);
    };
    size_t ncand = 0;
    for (int attempt = 0; attempt < 3; attempt++) {
        CUDA_TRY(cudaMemsetAsync(ws->d_counters, 0, 2 * sizeof(int), ws->stream));
        CUDA_TRY(cudaEventRecord(ws->ev0, ws->stream));
        if (plain) {
            // one launch per window over its own pieces: the per-window comparator
            int launches = 0;
            for (size_t w = 0; w + 1 < win_first.size(); w++) {
                size_t f = win_first[w], n = win_first[w + 1] - f;
                if (n == 0) continue;
                int grid = (int)std::min<int64_t>(((int64_t)n + best_l - 1) / best_l, max_ctas);
                CUDA_TRY(cudaMemsetAsync(ws->d_counters, 0, sizeof(int), ws->stream));
                CUDA_TRY(launch(f, n, grid));
                launches++;
            }
            ws->stats.kernel_launches += launches;
        } else {
            CUDA_TRY(launch(0, items.size(), ctas));
            ws->stats.kernel_launches += 1;
        }
        CUDA_TRY(cudaEventRecord(ws->ev1, ws->stream));
        CUDA_TRY(cudaMemcpyAsync(ws->h_counters, ws->d_counters, 2 * sizeof(int), cudaMemcpyDeviceToHost,
                                 ws->stream));
        CUDA_TRY(cudaStreamSynchronize(ws->stream));
        float ms = 0;
        cudaEventElapsedTime(&ms, ws->ev0, ws->ev1);
        ws->stats.kernel_ms += ms;
        ncand = (size_t)(unsigned)ws->h_counters[1];
        if (ncand <= ws->cands_cap) break;
        if ((rc = ensure_dev(&ws->d_cands, &ws->cands_cap, ncand + ncand / 4 + 1024))) return rc;
        if (attempt == 2) {
            set_error("candidate buffer overflow");
            return CMGPU_ENOSPACE;
        }
    }
    ws->stats.candidates = (int64_t)ncand;
    if ((rc = ensure_host_cands(ws, ncand + 1))) return rc;
    if (ncand)
        CUDA_TRY(cudaMemcpyAsync(ws->h_cands, ws->d_cands, ncand * sizeof(Cand), cudaMemcpyDeviceToHost,
                                 ws->stream));
    CUDA_TRY(cudaStreamSynchronize(ws->stream));

    // Order the cells by (window, j, d) in O(n): items ranked window by
    // window in column order, then a stable counting sort by item rank.  A
    // lane scans its item's columns in order, so an item's cells usually
    // arrive already in (j, d) order; a range that does not is sorted.
    std::vector<int32_t> rank(items.size());
    {
        std::vector<int32_t> ord(items.size());
        for (size_t x = 0; x < items.size(); x++) ord[x] = (int32_t)x;
        std::sort(ord.begin(), ord.end(), [&](int32_t a, int32_t b) {
            if (items[a].win != items[b].win) return items[a].win < items[b].win;
            return items[a].jreport < items[b].jreport;
        });
        for (size_t r = 0; r < ord.size(); r++) rank[ord[r]] = (int32_t)r;
    }
    std::vector<size_t> start(items.size() + 1, 0);
    for (size_t c = 0; c < ncand; c++) start[rank[ws->h_cands[c].item] + 1]++;
    for (size_t r = 0; r < items.size(); r++) start[r + 1] += start[r];
    std::vector<Cand> cs(ncand);
    {
        std::vector<size_t> pos(start.begin(), start.end() - 1);
        for (size_t c = 0; c < ncand; c++) {
            Cand x = ws->h_cands[c];
            const int32_t r = rank[x.item];
            x.item = items[x.item].win;
            cs[pos[r]++] = x;
        }
    }
    auto jd_less = [](const Cand &a, const Cand &b) { return a.j != b.j ? a.j < b.j : a.d < b.d; };
    for (size_t r = 0; r < items.size(); r++)
        if (!std::is_sorted(cs.begin() + start[r], cs.begin() + start[r + 1], jd_less))
            std::sort(cs.begin() + start[r], cs.begin() + start[r + 1], jd_less);
    if (cells_out) {
        *cells_out = cs;
        return CMGPU_OK;
    }
    // windows' ranges, and their frames on the host for null3
    struct Range {
        size_t b, e;
        int32_t win;
        const uint8_t *frame;
    };
    std::vector<Range> ranges;
    for (size_t k = 0; k < cs.size();) {
        size_t e = k;
        while (e < cs.size() && cs[e].item == cs[k].item) e++;
        ranges.push_back(Range{k, e, cs[k].item, nullptr});
        k = e;
    }
    std::vector<std::vector<uint8_t>> frame_bufs;
    if (do_null3) {
        if (!h_dsq) frame_bufs.resize(ranges.size());
        for (size_t r = 0; r < ranges.size(); r++) {
            const WinDesc &w = wins[ranges[r].win];
            if (h_dsq) {
                ranges[r].frame = h_dsq + w.off;
            } else {
                frame_bufs[r].resize((size_t)w.j0 + 2);
                CUDA_TRY(cudaMemcpy(frame_bufs[r].data(), d_dsq + w.off, (size_t)w.j0 + 1, cudaMemcpyDeviceToHost));
                ranges[r].frame = frame_bufs[r].data();
            }
        }
    }
    // report_hits_greedily + overlap removal per window: windows are
    // independent, so they are replayed on the host's cores
    auto replay = [&](size_t r) {
        const Range &g = ranges[r];
        report_window(m, semiring, cs.data() + g.b, g.e - g.b, g.frame, wins[g.win].i0, cutoff, do_null3,
                      hits_per_win[g.win]);
    };
    const size_t nthr = std::min<size_t>(ranges.size(), std::max(1u, std::thread::hardware_concurrency()));
    if (nthr <= 1 || cs.size() < (1u << 16)) {
        for (size_t r = 0; r < ranges.size(); r++) replay(r);
    } else {
        std::atomic<size_t> next{0};
        std::vector<std::thread> pool;
        for (size_t t = 0; t < nthr; t++)
            pool.emplace_back([&]() {
                for (size_t r; (r = next.fetch_add(1)) < ranges.size();) replay(r);
            });
        for (auto &th : pool) th.join();
    }
    (void)dsq_len;
    return CMGPU_OK;
}

static bool check_codes(const uint8_t *dsq, int32_t n);

// Copies a host residue buffer to the workspace.  frame=true: the buffer is
// one window frame, whose residues 1..len-2 are checked to be codes 0..17.
static int stage_dsq(cmgpu_workspace *ws, const uint8_t *h, int64_t len, bool frame = true) {
    if (frame && len >= 2 && !check_codes(h, (int32_t)(len - 2))) {
        set_error("residue code > 17 in the sequence");
        return CMGPU_EINVAL;
    }
    int rc = ensure_dev(&ws->d_dsq, &ws->dsq_cap, (size_t)len);
    if (rc) return rc;
    CUDA_TRY(cudaMemcpyAsync(ws->d_dsq, h, (size_t)len, cudaMemcpyHostToDevice, ws->stream));
    return CMGPU_OK;
}

static bool check_windows(const cmgpu_window *wins, int32_t nwin, int64_t dsq_len, const uint8_t *h_dsq) {
    for (int32_t k = 0; k < nwin; k++) {
        const cmgpu_window &w = wins[k];
        if (w.dsq_offset < 0 || w.i0 < 1 || w.j0 < w.i0 - 1) return false;
        if (w.dsq_offset + (int64_t)w.j0 + 1 > dsq_len) return false;
        if (h_dsq)
            for (int32_t x = w.i0; x <= w.j0; x++)
                if (h_dsq[w.dsq_offset + x] > 17) return false;
    }
    return true;
}

static bool check_codes(const uint8_t *dsq, int32_t n) {
    for (int32_t x = 1; x <= n; x++)
        if (dsq[x] > 17) return false;
    return true;
}

}  // namespace cmx

// ===========================================================================
// exported entry points
// ===========================================================================
extern "C" {

const char *cmgpu_last_error(void) { return cmx::g_err.c_str(); }
const char *cmgpu_version(void) { return "cmscan_gpu 0.1 (sm_100a)"; }

int cmgpu_model_upload(const cmgpu_cm *cm, int device, cmgpu_model **out) {
    if (!cm || !out) return CMGPU_EINVAL;
    *out = nullptr;
    std::unique_ptr<cmgpu_model> m(new cmgpu_model());
    m->device = device;
    if (!m->cm.load(cm)) {
        set_error("cmgpu_model_upload: inconsistent model arrays");
        return CMGPU_EINVAL;
    }
    CUDA_TRY(cudaSetDevice(device));
    std::vector<int32_t> t(LOGSUM_TBL);
    cmgpu_ilogsum_table(t.data(), LOGSUM_TBL);
    int nz = 0;
    for (int i = 0; i < LOGSUM_TBL; i++)
        if (t[i] != 0) nz = i + 1;
    // entries 0..nz-1, then zeros: the kernels index tbl[nz] (= 0) for the
    // ILogsum cases that add nothing and copy whole 32-bit words
    std::vector<uint16_t> t16(nz + 2, 0);
    for (int i = 0; i < nz; i++) t16[i] = (uint16_t)t[i];
    m->ilog_nz = nz;
    int rc = upload_vec(&m->ilog, t16);
    if (rc) return rc;
    m->flog.resize(LOGSUM_TBL);
    cmgpu_flogsum_table(m->flog.data(), LOGSUM_TBL);
    *out = m.release();
    return CMGPU_OK;
}

void cmgpu_model_free(cmgpu_model *m) { delete m; }

int cmgpu_workspace_create(int device, void *stream, cmgpu_workspace **out) {
    if (!out) return CMGPU_EINVAL;
    *out = nullptr;
    std::unique_ptr<cmgpu_workspace> ws(new cmgpu_workspace());
    ws->device = device;
    CUDA_TRY(cudaSetDevice(device));
    if (stream) {
        ws->stream = (cudaStream_t)stream;
    } else {
        CUDA_TRY(cudaStreamCreateWithFlags(&ws->stream, cudaStreamNonBlocking));
        ws->own_stream = true;
    }
    CUDA_TRY(cudaEventCreate(&ws->ev0));
    CUDA_TRY(cudaEventCreate(&ws->ev1));
    CUDA_TRY(cudaMalloc((void **)&ws->d_counters, 4 * sizeof(int)));
    CUDA_TRY(cudaMallocHost((void **)&ws->h_counters, 4 * sizeof(int)));
    cudaDeviceProp prop;
    CUDA_TRY(cudaGetDeviceProperties(&prop, device));
    ws->sm_count = prop.multiProcessorCount;
    *out = ws.release();
    return CMGPU_OK;
}

void cmgpu_workspace_free(cmgpu_workspace *ws) { delete ws; }

int cmgpu_workspace_stats(const cmgpu_workspace *ws, cmgpu_stats *out) {
    if (!ws || !out) return CMGPU_EINVAL;
    *out = ws->stats;
    return CMGPU_OK;
}

int cmgpu_workspace_set_kernel(cmgpu_workspace *ws, int kernel) {
    if (!ws || kernel < CMGPU_KERNEL_AUTO || kernel > CMGPU_KERNEL_SWEEP) return CMGPU_EINVAL;
    ws->kernel = kernel;
    return CMGPU_OK;
}

int cmgpu_workspace_set_shape(cmgpu_workspace *ws, int ctas_per_sm, int threads, int chunk, int lanes) {
    if (!ws) return CMGPU_EINVAL;
    if (threads != 0 && threads != 128 && threads != 256 && threads != 512) return CMGPU_EINVAL;
    if (lanes < 0 || lanes > MAX_LANES || ctas_per_sm < 0 || ctas_per_sm > 4) return CMGPU_EINVAL;
    ws->ctas_per_sm = ctas_per_sm;
    if (threads) ws->threads = threads;
    ws->chunk = chunk;
    ws->lanes = lanes;
    return CMGPU_OK;
}

static int finish_single(const std::vector<std::vector<cmgpu_hit>> &hpw, cmgpu_hit *hits, int32_t cap,
                         int32_t *n_out) {
    size_t n = 0;
    for (auto &v : hpw) n += v.size();
    *n_out = (int32_t)n;
    if ((int64_t)n > cap) {
        set_error("output array too small");
        return CMGPU_EOVERFLOW;
    }
    size_t o = 0;
    for (auto &v : hpw)
        for (auto &h : v) hits[o++] = h;
    return CMGPU_OK;
}

int cmgpu_qdb_scan(const cmgpu_model *mc, cmgpu_workspace *ws, int semiring, int qdbidx, const uint8_t *dsq,
                   int32_t n, int32_t i0, int32_t j0, float cutoff, int do_null3, cmgpu_hit *hits, int32_t cap,
                   int32_t *n_out) {
    cmgpu_model *m = const_cast<cmgpu_model *>(mc);
    if (!m || !ws || !dsq || !n_out || n < 0 || i0 < 1 || j0 > n || (cap > 0 && !hits)) return CMGPU_EINVAL;
    *n_out = 0;
    int rc = stage_dsq(ws, dsq, (int64_t)n + 2);
    if (rc) return rc;
    std::vector<WinDesc> wins{{0, i0, j0}};
    std::vector<std::vector<cmgpu_hit>> hpw;
    rc = run_scan(m, ws, semiring, qdbidx, ws->d_dsq, dsq, (int64_t)n + 2, wins, cutoff, do_null3, false, hpw);
    if (rc) return rc;
    return finish_single(hpw, hits, cap, n_out);
}

int cmgpu_qdb_scan_cells(const cmgpu_model *mc, cmgpu_workspace *ws, int semiring, int qdbidx, const uint8_t *dsq,
                         int32_t n, int32_t i0, int32_t j0, float cutoff, int32_t *cj, int32_t *cd, float *csc,
                         int32_t cap, int32_t *n_out) {
    cmgpu_model *m = const_cast<cmgpu_model *>(mc);
    if (!m || !ws || !dsq || !n_out || n < 0 || i0 < 1 || j0 > n || (cap > 0 && (!cj || !cd || !csc)))
        return CMGPU_EINVAL;
    *n_out = 0;
    int rc = stage_dsq(ws, dsq, (int64_t)n + 2);
    if (rc) return rc;
    std::vector<WinDesc> wins{{0, i0, j0}};
    std::vector<std::vector<cmgpu_hit>> hpw;
    std::vector<Cand> cells;
    rc = run_scan(m, ws, semiring, qdbidx, ws->d_dsq, dsq, (int64_t)n + 2, wins, cutoff, 0, false, hpw, &cells);
    if (rc) return rc;
    *n_out = (int32_t)cells.size();
    if ((int64_t)cells.size() > cap) {
        set_error("output array too small");
        return CMGPU_EOVERFLOW;
    }
    for (size_t k = 0; k < cells.size(); k++) {
        cj[k] = cells[k].j;
        cd[k] = cells[k].d;
        csc[k] = raw_bits(semiring, cells[k].raw);
    }
    return CMGPU_OK;
}

int cmgpu_cyk_seq_filter(const cmgpu_model *mc, cmgpu_workspace *ws, const uint8_t *dsq, int32_t n, float cutoff,
                         int do_null3, cmgpu_envelope *envs, int32_t cap, int32_t *n_out) {
    cmgpu_model *m = const_cast<cmgpu_model *>(mc);
    if (!m || !ws || !dsq || !n_out || n < 0 || (cap > 0 && !envs)) return CMGPU_EINVAL;
    *n_out = 0;
    if (n == 0) return CMGPU_OK;
    int rc = stage_dsq(ws, dsq, (int64_t)n + 2);
    if (rc) return rc;
    std::vector<WinDesc> wins{{0, 1, n}};
    std::vector<std::vector<cmgpu_hit>> hpw;
    rc = run_scan(m, ws, CMGPU_CYK_F32, CMGPU_QDB1, ws->d_dsq, dsq, (int64_t)n + 2, wins, cutoff, do_null3, false,
                  hpw);
    if (rc) return rc;
    // pad each hit by W-1 and merge (src/cm_nohmm.rs:858-888)
    const int W = m->cm.view.W;
    std::vector<std::pair<int32_t, int32_t>> pad;
    for (auto &h : hpw[0]) pad.push_back({std::max(1, h.j - (W - 1)), std::min(n, h.i + (W - 1))});
    std::sort(pad.begin(), pad.end(), [](const std::pair<int32_t, int32_t> &a, const std::pair<int32_t, int32_t> &b) {
        if (a.second != b.second) return a.second < b.second;
        return a.first < b.first;
    });
    std::vector<cmgpu_envelope> out;
    size_t h = 0;
    while (h < pad.size()) {
        int32_t iw = pad[h].first, jw = pad[h].second;
        while (h + 1 < pad.size() && pad[h + 1].first <= jw) {
            h++;
            jw = std::max(jw, pad[h].second);
        }
        out.push_back(cmgpu_envelope{iw, jw});
        h++;
    }
    *n_out = (int32_t)out.size();
    if ((int64_t)out.size() > cap) {
        set_error("output array too small");
        return CMGPU_EOVERFLOW;
    }
    std::copy(out.begin(), out.end(), envs);
    return CMGPU_OK;
}

int cmgpu_final_stage_inside_opt(const cmgpu_model *mc, cmgpu_workspace *ws, const uint8_t *dsq, int32_t n,
                                 const cmgpu_envelope *envs, int32_t nenv, float cutoff, int do_null3, int nonbanded,
                                 cmgpu_hit *hits, int32_t cap, int32_t *n_out) {
    cmgpu_model *m = const_cast<cmgpu_model *>(mc);
    if (!m || !ws || !dsq || !n_out || n < 0 || nenv < 0 || (nenv > 0 && !envs) || (cap > 0 && !hits))
        return CMGPU_EINVAL;
    *n_out = 0;
    std::vector<WinDesc> wins;
    for (int32_t k = 0; k < nenv; k++) {
        if (envs[k].start < 1 || envs[k].end > n) {
            set_error("envelope outside the sequence");
            return CMGPU_EINVAL;
        }
        wins.push_back(WinDesc{0, envs[k].start, envs[k].end});
    }
    if (wins.empty()) return CMGPU_OK;
    int rc = stage_dsq(ws, dsq, (int64_t)n + 2);
    if (rc) return rc;
    std::vector<std::vector<cmgpu_hit>> hpw;
    rc = run_scan(m, ws, CMGPU_INSIDE_I32, nonbanded ? CMGPU_NOQDB : CMGPU_QDB2, ws->d_dsq, dsq, (int64_t)n + 2,
                  wins, cutoff, do_null3, false, hpw);
    if (rc) return rc;
    return finish_single(hpw, hits, cap, n_out);
}

static int batch_common(const cmgpu_model *mc, cmgpu_workspace *ws, int semiring, int qdbidx, const uint8_t *h_dsq,
                        const uint8_t *d_dsq, int64_t dsq_len, const cmgpu_window *wins, int32_t nwin, float cutoff,
                        int do_null3, bool plain, cmgpu_batch_hit *hits, int32_t cap, int32_t *n_out,
                        bool calib = false) {
    cmgpu_model *m = const_cast<cmgpu_model *>(mc);
    if (!m || !ws || !n_out || nwin < 0 || (nwin > 0 && !wins) || (cap > 0 && !hits)) return CMGPU_EINVAL;
    *n_out = 0;
    if (!check_windows(wins, nwin, dsq_len, h_dsq)) {
        set_error("window outside the residue buffer, or residue code > 17");
        return CMGPU_EINVAL;
    }
    if (nwin == 0) return CMGPU_OK;
    std::vector<WinDesc> wv;
    for (int32_t k = 0; k < nwin; k++) wv.push_back(WinDesc{wins[k].dsq_offset, wins[k].i0, wins[k].j0});
    int rc;
    if (h_dsq) {
        if ((rc = stage_dsq(ws, h_dsq, dsq_len, false))) return rc;
        d_dsq = ws->d_dsq;
    }
    std::vector<std::vector<cmgpu_hit>> hpw;
    rc = run_scan(m, ws, semiring, qdbidx, d_dsq, h_dsq, dsq_len, wv, cutoff, do_null3, plain, hpw, nullptr, calib);
    if (rc) return rc;
    size_t n = 0;
    for (auto &v : hpw) n += v.size();
    *n_out = (int32_t)n;
    if ((int64_t)n > cap) {
        set_error("output array too small");
        return CMGPU_EOVERFLOW;
    }
    size_t o = 0;
    for (size_t w = 0; w < hpw.size(); w++)
        for (auto &h : hpw[w]) hits[o++] = cmgpu_batch_hit{(int32_t)w, h.i, h.j, h.score, h.bias};
    return CMGPU_OK;
}

int cmgpu_scan_batch(const cmgpu_model *m, cmgpu_workspace *ws, int semiring, int qdbidx, const uint8_t *dsq_all,
                     int64_t dsq_len, const cmgpu_window *wins, int32_t nwin, float cutoff, int do_null3,
                     cmgpu_batch_hit *hits, int32_t cap, int32_t *n_out) {
    if (!dsq_all) return CMGPU_EINVAL;
    return batch_common(m, ws, semiring, qdbidx, dsq_all, nullptr, dsq_len, wins, nwin, cutoff, do_null3, false, hits,
                        cap, n_out);
}

int cmgpu_scan_batch_device(const cmgpu_model *m, cmgpu_workspace *ws, int semiring, int qdbidx,
                            const uint8_t *d_dsq_all, int64_t dsq_len, const cmgpu_window *wins, int32_t nwin,
                            float cutoff, int do_null3, cmgpu_batch_hit *hits, int32_t cap, int32_t *n_out) {
    if (!d_dsq_all) return CMGPU_EINVAL;
    return batch_common(m, ws, semiring, qdbidx, nullptr, d_dsq_all, dsq_len, wins, nwin, cutoff, do_null3, false,
                        hits, cap, n_out);
}

int cmgpu_scan_plain(const cmgpu_model *m, cmgpu_workspace *ws, int semiring, int qdbidx, const uint8_t *dsq_all,
                     int64_t dsq_len, const cmgpu_window *wins, int32_t nwin, float cutoff, int do_null3,
                     cmgpu_batch_hit *hits, int32_t cap, int32_t *n_out) {
    if (!dsq_all) return CMGPU_EINVAL;
    return batch_common(m, ws, semiring, qdbidx, dsq_all, nullptr, dsq_len, wins, nwin, cutoff, do_null3, true, hits,
                        cap, n_out);
}

// collect_scores's scan (src/cm_calibrate.rs:953-989): every window with
// cutoff -inf, local begins in bit-score order
int cmgpu_calibrate_scan_batch(const cmgpu_model *m, cmgpu_workspace *ws, int semiring, int qdbidx,
                               const uint8_t *dsq_all, int64_t dsq_len, const cmgpu_window *wins, int32_t nwin,
                               int do_null3, cmgpu_batch_hit *hits, int32_t cap, int32_t *n_out) {
    if (!dsq_all) return CMGPU_EINVAL;
    if (ws && ws->kernel == CMGPU_KERNEL_SWEEP) {
        set_error("cmcalibrate's scan runs on the level kernel only");
        return CMGPU_EINVAL;
    }
    return batch_common(m, ws, semiring, qdbidx, dsq_all, nullptr, dsq_len, wins, nwin, -INFINITY, do_null3, false,
                        hits, cap, n_out, true);
}

}  // extern "C"
