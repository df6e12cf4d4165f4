// Launch interface between the host orchestration (capi.cpp) and the
// node-sweep scan kernel (sweep_scan.cu).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

#include "qdb_kernel.h"
#include "sweep_plan.h"

namespace cmx {

constexpr int SW_MAX_WARPS = 12;  // warps (work items) per CTA

// Shared-memory layout of one CTA, in 32-bit words.  Model tables first,
// then one region per warp.
struct SwLayout {
    int st, kid, tsc, endsc, init0, bsv, escc, el, tbl, nodes, io, bifs;
    int warp0;   // first per-warp region
    int wwords;  // words per warp region: node buffers, previous-column
                 // buffer, BEGR rows, local-begin row, residue ring
    int ring_len;
    int64_t words;
};

struct SweepParams {
    // plan (device memory)
    const SwState *st;
    const uint8_t *kid;
    const SwNode *nodes;
    const SwIO *io;
    const SwBif *bifs;
    const uint32_t *tsc, *endsc, *init0, *bsv, *esc, *esc_c, *el_sca;
    const uint16_t *ilog;
    int ilog_nz;
    int M, W, S, RW, nnodes, nio, nbif, n_esc_c;
    int local;
    int inside;
    // work
    const uint8_t *dsq;
    const WorkItem *items;
    int nitems;
    int item_base;
    int *next_item;
    Cand *cands;
    int cand_cap;
    int *cand_count;
    float cutoff;
    // per-warp global memory: deck slots, then the BEGL rings
    uint32_t *gmem;
    int64_t gstride;     // words per warp
    int64_t deck_words;  // words of deck slots per warp
    int warps;           // per CTA
    SwLayout lay;
};

SwLayout sweep_layout(const SweepParams &p, int warps);
int sweep_occupancy(const SweepParams &p, int threads);
cudaError_t sweep_launch(const SweepParams &p, int ctas, cudaStream_t s);

}  // namespace cmx
