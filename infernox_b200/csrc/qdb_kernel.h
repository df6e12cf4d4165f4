// Launch interface between the host orchestration (capi.cpp) and the scan
// kernel (qdb_scan.cu).
#pragma once
#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>

#include "qdb_plan.h"

namespace cmx {

constexpr int IL_KMAX = 8;     // IL cells per lane kept in registers (W <= 255)
constexpr int COL_BLOCK = 32;  // columns a lane advances between refills
constexpr int MAX_LANES = 16;  // work items one CTA scans side by side

// A piece of one window: columns jstart..jend are scanned, candidates are
// emitted for columns >= jreport (the first W-1 are warm-up).
struct WorkItem {
    int64_t dsq_off;  // offset of the window frame in the residue buffer
    int32_t jstart, jend, jreport, win;
};

// A reportable cell: bestsc(j, d) >= cutoff, raw value in the semiring.
struct Cand {
    int32_t item, j, d;
    uint32_t raw;
};

// Shared-memory layout of one CTA, in 32-bit words from the start of the
// dynamic shared memory.  Computed once on the host (scan_layout).
struct SmemLayout {
    int el, tbl, info, wb, cb, tsc, endsc, escc, chunks, lvl, begin, beginsc, ring, lane, deck;
    int bsv, bmax;     // fused local begins: per-state begin score, per-lane ROOT row
    int prow;          // report pre-filter: per-lane ROOT row of raw values
    int ring_len;      // residues per lane ring (power of two >= W + 64)
    int64_t words;     // total
};

struct ScanParams {
    // plan (device, global memory; copied to shared memory at kernel start)
    const StateDev *states;
    const int32_t *wb, *cb;
    const ChunkDev *chunks;
    const int32_t *level_start;
    int nlev, nchunks;
    const uint32_t *tsc, *endsc, *esc, *el_sca, *esc_c;
    int n_esc_c;
    const BeginDev *begins;
    const uint32_t *beginsc;
    int nbegin;
    // fused local begins (integer Inside): every begin state's cells post
    // cell + beginsc to a per-lane ROOT row with an atomic max
    int fuse_begin;
    const uint32_t *beginsc_all;  // [M], -INFTY where no local begin
    const int32_t *init_off;
    const uint32_t *init_val;
    int ninit;
    int M, W;
    int root_dn, root_dxcap, root_cnum;
    int local;
    int inside;
    int64_t deck_elems;
    // ILogsum table up to its last nonzero entry
    const uint16_t *ilog;
    int ilog_nz;
    // work
    const uint8_t *dsq;
    const WorkItem *items;
    int nitems;
    int item_base;  // added to the item index recorded in candidates
    int *next_item;
    Cand *cands;
    int cand_cap;
    int *cand_count;
    float cutoff;
    // per-state tables read from global memory instead of shared memory
    // (models whose tables would not leave room for a lane)
    int tables_global;
    // lanes per CTA and deck placement
    // cmcalibrate's scan (src/cm_calibrate.rs:441-780): local begins are
    // compared in bits, so -INFTY orders below every other integer value
    // (scorify maps it to IMPOSSIBLE, and nothing else)
    int begin_key;
    // report pre-filter: of the ROOT cells of a column only those that the
    // greedy report (with null3) could report are emitted; the rest can be
    // neither reported nor raise the running maximum of reported scores
    int prefilter;
    int do_null3;
    float pf_null[4];
    float pf_omega;
    int lanes;
    int deck_smem;
    uint32_t *deck_global;  // when !deck_smem: [ctas][lanes][deck_stride]
    int64_t deck_stride;
    SmemLayout lay;
};

SmemLayout scan_layout(const ScanParams &p, int lanes, bool deck_smem);
int scan_occupancy(const ScanParams &p, int threads);
cudaError_t scan_launch(const ScanParams &p, int ctas, int threads, cudaStream_t s);

}  // namespace cmx
