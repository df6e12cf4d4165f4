// cmgpu_qdb_scan_noalloc: the window scan of cmgpu_qdb_scan for callers that
// must not allocate device memory.
//
// Who needs it: a process whose device memory is owned by someone else -- a
// framework's caching allocator that has reserved most of the GPU, or a
// server that gives each tenant a fixed device-memory budget -- where a raw
// cudaMalloc fails or escapes the accounting; and a process that runs other
// streams on the same GPU and cannot accept the device-wide synchronisation
// that cudaFree implies.  The regular entry points grow per-workspace
// buffers with cudaMalloc and cudaFree; this one never calls either.
//
// Where its scratch lives: one file-scope `static __device__` array of
// NOALLOC_SCRATCH_BYTES (16 MiB).  Every GPU that loads this library reserves
// it when the module is loaded, and keeps it until the process exits.  The
// scan's per-call data -- a copy of the scan plan, the residues, the work
// items, the two queue counters, the reportable-cell buffer and, when the
// decks do not fit in shared memory, the decks -- is placed inside it.  A
// request that does not fit is rejected with CMGPU_ENOSPACE before any copy.
//
// Set-up: the host needs the array's device address (its name in host code
// is only a host-side stand-in).  The first call on a device looks the
// address up once with cudaGetSymbolAddress, with that device current.
//
// Blocking: the call copies its inputs, launches the scan and waits for its
// stream (it reads the cell count back to size the result), so it returns
// with the scan finished.  The calling thread's current device is the same on
// return as on entry.
//
// Sharing: all calls on one device use the same array, which keeps whatever
// the previous call left there.  The counters are cleared on every call and
// every deck is refilled by the kernel before use; calls that overlap on the
// GPU (different streams, or different host threads without ordering) race
// on the array, so the caller must serialise them.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <vector>

#include "model_internal.h"

namespace cmx {

constexpr size_t NOALLOC_SCRATCH_BYTES = (size_t)16 << 20;
constexpr int NOALLOC_MAX_DEVICES = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

static std::mutex g_noalloc_mu;
static unsigned char *g_noalloc_ptr[NOALLOC_MAX_DEVICES];

// Device address of the scratch array on `device` (made current by the
// caller), looked up once per device.
static int noalloc_scratch(int device, unsigned char **out) {
    if (device < 0 || device >= NOALLOC_MAX_DEVICES) {
        set_error("cmgpu_qdb_scan_noalloc: device index out of range");
        return CMGPU_EINVAL;
    }
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[device]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            set_error(std::string("cmgpu_qdb_scan_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
            return CMGPU_EDEVICE;
        }
        g_noalloc_ptr[device] = static_cast<unsigned char *>(p);
    }
    *out = g_noalloc_ptr[device];
    return CMGPU_OK;
}

// Makes `device` current for the life of the guard and restores the caller's
// current device afterwards.
struct DeviceGuard {
    int prev = -1;
    cudaError_t err = cudaSuccess;
    explicit DeviceGuard(int device) {
        err = cudaGetDevice(&prev);
        if (err == cudaSuccess && prev != device) err = cudaSetDevice(device);
    }
    ~DeviceGuard() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

// The model's host scan plan for (semiring, qdbidx), built on first use and
// kept with the model (host memory only).
static const Plan *noalloc_plan(const cmgpu_model *m, int semiring, int qdbidx) {
    std::lock_guard<std::mutex> lk(m->noalloc_mu);
    const int key = semiring * 8 + qdbidx;
    auto it = m->noalloc_plans.find(key);
    if (it != m->noalloc_plans.end()) return it->second.get();
    std::unique_ptr<Plan> pl(new Plan());
    if (!build_plan(&m->cm.view, semiring, qdbidx, *pl)) return nullptr;
    const Plan *out = pl.get();
    m->noalloc_plans[key] = std::move(pl);
    return out;
}

// Bump allocator over a region of the scratch array (offsets only; nothing
// is allocated).
struct Carve {
    size_t used = 0, cap = 0;
    bool ok = true;
    size_t take(size_t bytes) {
        size_t off = (used + 255) & ~(size_t)255;
        if (off + bytes > cap) {
            ok = false;
            return 0;
        }
        used = off + bytes;
        return off;
    }
};

}  // namespace cmx

using namespace cmx;

#define NA_TRY(call)                                                                            \
    do {                                                                                        \
        cudaError_t e_ = (call);                                                                \
        if (e_ != cudaSuccess) {                                                                \
            set_error(std::string("cmgpu_qdb_scan_noalloc: ") + #call + ": " + cudaGetErrorString(e_)); \
            return CMGPU_EDEVICE;                                                               \
        }                                                                                       \
    } while (0)

extern "C" int cmgpu_qdb_scan_noalloc(const cmgpu_model *m, void *stream_ptr, int semiring, int qdbidx,
                                      const uint8_t *dsq, int32_t n, int32_t i0, int32_t j0, float cutoff,
                                      int do_null3, cmgpu_hit *hits, int32_t cap, int32_t *n_out) {
    if (!m || !dsq || !n_out || n < 0 || i0 < 1 || j0 > n || (cap > 0 && !hits) ||
        (semiring != CMGPU_CYK_F32 && semiring != CMGPU_INSIDE_I32) || qdbidx < 0 || qdbidx > 2) {
        set_error("cmgpu_qdb_scan_noalloc: bad arguments");
        return CMGPU_EINVAL;
    }
    *n_out = 0;
    for (int32_t x = 1; x <= n; x++)
        if (dsq[x] > 17) {
            set_error("cmgpu_qdb_scan_noalloc: residue code > 17 in the sequence");
            return CMGPU_EINVAL;
        }
    if (j0 < i0) return CMGPU_OK;
    cudaStream_t st = (cudaStream_t)stream_ptr;
    DeviceGuard dg(m->device);
    NA_TRY(dg.err);
    unsigned char *scratch = nullptr;
    int rc = noalloc_scratch(m->device, &scratch);
    if (rc) return rc;

    // scan plan: built on the host once per model, copied into the scratch array
    const Plan *plp = noalloc_plan(m, semiring, qdbidx);
    if (!plp) {
        set_error(std::string("cmgpu_qdb_scan_noalloc: scan plan: ") + cmgpu_last_error());
        return CMGPU_EINVAL;
    }
    const Plan &pl = *plp;
    const int W = pl.W;

    // work items: the window in pieces of `chunk` reported columns
    int dev_sms = 148;
    NA_TRY(cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, m->device));
    const int64_t L = (int64_t)j0 - i0 + 1;
    int64_t chunk = std::max<int64_t>(4 * (int64_t)W, L / ((int64_t)dev_sms * 4) + 1);
    std::vector<WorkItem> items;
    for (int64_t r0 = i0; r0 <= j0; r0 += chunk) {
        int64_t r1 = std::min<int64_t>(j0, r0 + chunk - 1);
        int64_t js = std::max<int64_t>(i0, r0 - (W - 1));
        items.push_back(WorkItem{0, (int32_t)js, (int32_t)r1, (int32_t)r0, 0});
    }

    // layout of this call inside the scratch array
    Carve cv;
    cv.cap = NOALLOC_SCRATCH_BYTES;
    auto put = [&](size_t bytes) -> size_t { return cv.take(std::max<size_t>(bytes, 4)); };
    const size_t o_states = put(pl.states.size() * sizeof(StateDev));
    const size_t o_wb = put(pl.wb.size() * 4);
    const size_t o_cb = put(pl.cb.size() * 4);
    const size_t o_chunks = put(pl.chunks.size() * sizeof(ChunkDev));
    const size_t o_lvl = put(pl.level_start.size() * 4);
    const size_t o_tsc = put(pl.tsc.size() * 4);
    const size_t o_endsc = put(pl.endsc.size() * 4);
    const size_t o_esc = put(pl.esc.size() * 4);
    const size_t o_el = put(pl.el_sca.size() * 4);
    const size_t o_escc = put(pl.esc_c.size() * 4);
    const size_t o_begins = put(pl.begins.size() * sizeof(BeginDev));
    const size_t o_beginsc = put(pl.beginsc.size() * 4);
    const size_t o_ioff = put(pl.init_off.size() * 4);
    const size_t o_ival = put(pl.init_val.size() * 4);
    const size_t o_dsq = put((size_t)n + 2);
    const size_t o_items = put(items.size() * sizeof(WorkItem));
    const size_t o_cnt = put(2 * sizeof(int));
    if (!cv.ok) {
        set_error("cmgpu_qdb_scan_noalloc: model plus sequence exceed the 16 MiB scratch array");
        return CMGPU_ENOSPACE;
    }

    ScanParams sp{};
    auto at = [&](size_t off) { return scratch + off; };
    sp.states = reinterpret_cast<const StateDev *>(at(o_states));
    sp.wb = reinterpret_cast<const int32_t *>(at(o_wb));
    sp.cb = reinterpret_cast<const int32_t *>(at(o_cb));
    sp.chunks = reinterpret_cast<const ChunkDev *>(at(o_chunks));
    sp.level_start = reinterpret_cast<const int32_t *>(at(o_lvl));
    sp.nlev = (int)pl.level_start.size() - 1;
    sp.nchunks = (int)pl.chunks.size();
    sp.tsc = reinterpret_cast<const uint32_t *>(at(o_tsc));
    sp.endsc = reinterpret_cast<const uint32_t *>(at(o_endsc));
    sp.esc = reinterpret_cast<const uint32_t *>(at(o_esc));
    sp.el_sca = reinterpret_cast<const uint32_t *>(at(o_el));
    sp.esc_c = reinterpret_cast<const uint32_t *>(at(o_escc));
    sp.n_esc_c = (int)pl.esc_c.size();
    sp.begins = reinterpret_cast<const BeginDev *>(at(o_begins));
    sp.beginsc = reinterpret_cast<const uint32_t *>(at(o_beginsc));
    sp.nbegin = (int)pl.begins.size();
    sp.init_off = reinterpret_cast<const int32_t *>(at(o_ioff));
    sp.init_val = reinterpret_cast<const uint32_t *>(at(o_ival));
    sp.ninit = (int)pl.init_off.size();
    sp.M = pl.M;
    sp.W = W;
    sp.root_dn = pl.root_dn;
    sp.root_dxcap = pl.root_dxcap;
    sp.root_cnum = pl.root_cnum;
    sp.local = pl.local ? 1 : 0;
    sp.inside = semiring == CMGPU_INSIDE_I32;
    sp.deck_elems = pl.deck_elems;
    sp.ilog = m->ilog;
    sp.ilog_nz = m->ilog_nz;
    sp.dsq = at(o_dsq);
    sp.items = reinterpret_cast<const WorkItem *>(at(o_items));
    sp.nitems = (int)items.size();
    sp.item_base = 0;
    sp.next_item = reinterpret_cast<int *>(at(o_cnt));
    sp.cand_count = sp.next_item + 1;
    sp.cutoff = cutoff;

    // launch shape: decks in shared memory when one lane fits, else in the
    // scratch array beside the cell buffer
    const int threads = 512;
    const size_t SMEM_CAP = 227 * 1024 - 1024;
    int lanes = 0;
    for (int t = MAX_LANES; t >= 1; t--)
        if ((size_t)scan_layout(sp, t, true).words * 4 <= SMEM_CAP) {
            lanes = t;
            break;
        }
    bool deck_smem = lanes > 0;
    int ctas = 0;
    size_t o_deck = 0, stride = ((size_t)pl.deck_elems + 31) & ~(size_t)31;
    if (deck_smem) {
        ctas = (int)std::min<int64_t>(((int64_t)items.size() + lanes - 1) / lanes, dev_sms);
    } else {
        lanes = 1;
        // decks take at most half of what is left; the rest holds cells
        size_t left = cv.cap - ((cv.used + 255) & ~(size_t)255);
        size_t per_cta = stride * 4 * (size_t)lanes;
        int fit = (int)std::min<size_t>(left / 2 / std::max<size_t>(per_cta, 1), (size_t)dev_sms);
        if (fit < 1) {
            set_error("cmgpu_qdb_scan_noalloc: the model's decks exceed the 16 MiB scratch array");
            return CMGPU_ENOSPACE;
        }
        ctas = (int)std::min<int64_t>((int64_t)items.size(), fit);
        o_deck = cv.take(per_cta * (size_t)ctas);
    }
    size_t left = cv.cap - ((cv.used + 255) & ~(size_t)255);
    size_t cand_cap = left / sizeof(Cand);
    size_t o_cands = cv.take(cand_cap * sizeof(Cand));
    if (!cv.ok || cand_cap < 1) {
        set_error("cmgpu_qdb_scan_noalloc: no room left for reportable cells in the scratch array");
        return CMGPU_ENOSPACE;
    }
    sp.lanes = lanes;
    sp.deck_smem = deck_smem ? 1 : 0;
    sp.deck_global = deck_smem ? nullptr : reinterpret_cast<uint32_t *>(at(o_deck));
    sp.deck_stride = (int64_t)stride;
    sp.cands = reinterpret_cast<Cand *>(at(o_cands));
    sp.cand_cap = (int)std::min<size_t>(cand_cap, (size_t)INT32_MAX);
    sp.lay = scan_layout(sp, lanes, deck_smem);
    if (scan_occupancy(sp, threads) < 1) {
        set_error("cmgpu_qdb_scan_noalloc: scan kernel cannot be resident with this shape");
        return CMGPU_EDEVICE;
    }

    // inputs into the scratch array; the queue and cell counters start at zero
    auto h2d = [&](size_t off, const void *src, size_t bytes) -> cudaError_t {
        if (bytes == 0) return cudaSuccess;
        return cudaMemcpyAsync(at(off), src, bytes, cudaMemcpyHostToDevice, st);
    };
    NA_TRY(h2d(o_states, pl.states.data(), pl.states.size() * sizeof(StateDev)));
    NA_TRY(h2d(o_wb, pl.wb.data(), pl.wb.size() * 4));
    NA_TRY(h2d(o_cb, pl.cb.data(), pl.cb.size() * 4));
    NA_TRY(h2d(o_chunks, pl.chunks.data(), pl.chunks.size() * sizeof(ChunkDev)));
    NA_TRY(h2d(o_lvl, pl.level_start.data(), pl.level_start.size() * 4));
    NA_TRY(h2d(o_tsc, pl.tsc.data(), pl.tsc.size() * 4));
    NA_TRY(h2d(o_endsc, pl.endsc.data(), pl.endsc.size() * 4));
    NA_TRY(h2d(o_esc, pl.esc.data(), pl.esc.size() * 4));
    NA_TRY(h2d(o_el, pl.el_sca.data(), pl.el_sca.size() * 4));
    NA_TRY(h2d(o_escc, pl.esc_c.data(), pl.esc_c.size() * 4));
    NA_TRY(h2d(o_begins, pl.begins.data(), pl.begins.size() * sizeof(BeginDev)));
    NA_TRY(h2d(o_beginsc, pl.beginsc.data(), pl.beginsc.size() * 4));
    NA_TRY(h2d(o_ioff, pl.init_off.data(), pl.init_off.size() * 4));
    NA_TRY(h2d(o_ival, pl.init_val.data(), pl.init_val.size() * 4));
    NA_TRY(h2d(o_dsq, dsq, (size_t)n + 2));
    NA_TRY(h2d(o_items, items.data(), items.size() * sizeof(WorkItem)));
    NA_TRY(cudaMemsetAsync(at(o_cnt), 0, 2 * sizeof(int), st));
    NA_TRY(scan_launch(sp, ctas, threads, st));
    int counters[2] = {0, 0};
    NA_TRY(cudaMemcpyAsync(counters, at(o_cnt), sizeof(counters), cudaMemcpyDeviceToHost, st));
    NA_TRY(cudaStreamSynchronize(st));
    const size_t ncand = (size_t)(unsigned)counters[1];
    if (ncand > cand_cap) {
        set_error("cmgpu_qdb_scan_noalloc: reportable cells exceed the room left in the scratch array; "
                  "raise the cutoff or scan a shorter window");
        return CMGPU_ENOSPACE;
    }
    std::vector<Cand> cs(ncand);
    if (ncand) {
        NA_TRY(cudaMemcpyAsync(cs.data(), at(o_cands), ncand * sizeof(Cand), cudaMemcpyDeviceToHost, st));
        NA_TRY(cudaStreamSynchronize(st));
    }
    std::sort(cs.begin(), cs.end(), [](const Cand &a, const Cand &b) {
        if (a.j != b.j) return a.j < b.j;
        return a.d < b.d;
    });
    std::vector<cmgpu_hit> out;
    report_window(m, semiring, cs.data(), cs.size(), dsq, i0, cutoff, do_null3, out);
    *n_out = (int32_t)out.size();
    if ((int64_t)out.size() > cap) {
        set_error("output array too small");
        return CMGPU_EOVERFLOW;
    }
    std::copy(out.begin(), out.end(), hits);
    return CMGPU_OK;
}
