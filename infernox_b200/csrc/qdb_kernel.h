// Launch interface between the host orchestration (capi.cpp) and the scan
// kernel (qdb_scan.cu).
#pragma once
#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>

#include "qdb_plan.h"

namespace cmx {

constexpr int IL_KMAX = 8;  // IL cells per lane kept in registers (W <= 255)

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

struct ScanParams {
    // plan (device)
    const StateDev *states;
    const ChunkDev *chunks;
    const int32_t *level_start;
    int nlev;
    const uint32_t *tsc, *init0, *endsc, *beginsc, *esc, *el_sca;
    const int32_t *begin_states;
    int nbegin;
    int M, W;
    int root_dn, root_dxcap, root_cfirst, root_cnum;
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
    // global deck fallback
    uint32_t *deck_global;
    int64_t deck_stride;
};

size_t scan_smem_bytes(const ScanParams &p, bool deck_smem);
int scan_occupancy(const ScanParams &p, bool deck_smem, int threads);
cudaError_t scan_launch(const ScanParams &p, bool deck_smem, int ctas, int threads, cudaStream_t s);

}  // namespace cmx
