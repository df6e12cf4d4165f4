// Host-side report of the truncated scanners, shared by the HMM-banded
// (hb_scan.cu) and the QDB / non-banded (trq_scan.cu) kernels: both emit the
// reportable cells of a window as TrCand, and the host replays the
// reference's greedy truncated report on them.
#pragma once
#include <cstdint>
#include <vector>

#include "model_internal.h"

namespace cmx {
namespace hb {
// marginal alignment modes (TRMODE_T/R/L/J/UNKNOWN, src/cm_dpsearch_trunc.rs)
enum { TRM_T = 0, TRM_R = 1, TRM_L = 2, TRM_J = 3, TRM_UNKNOWN = 4 };

// one reportable cell: window (or envelope) index, end j, length d, best
// truncated-begin score, its mode and entry state
struct TrCand {
    int32_t env, j, d;
    float sc;
    int32_t mode, root;
};
}  // namespace hb

struct TrCtx {
    const cmgpu_tr_tables *tt;
    int pass_idx, local;
};

// allow_truncation (src/cm_dpsearch_trunc.rs:2376-2440)
bool allow_trunc(const TrCtx &c, int64_t start, int64_t stop, int64_t i0, int64_t j0, int mode, int b);

// report_hits_greedily (src/cm_dpsearch_trunc.rs:2322-2374) over the
// reportable cells of one window, sorted by (j, d), with null3; then the
// overlap removal (:2470); appends the kept hits to `out`.
void tr_report(const cmgpu_model *m, const TrCtx &cx, const hb::TrCand *c, size_t n, const uint8_t *dsq, int32_t i0,
               int32_t j0, float cutoff, int do_null3, std::vector<cmgpu_tr_hit> &out);
}  // namespace cmx
