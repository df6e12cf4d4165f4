// Device-side plan of one configured CM for one (semiring, band set): the
// per-state metadata, the compact deck layout and the level schedule the
// scan kernel walks every column.  Built on the host (qdb_plan.cpp) and
// copied to device memory once per model.
#pragma once
#include <cstdint>
#include <vector>

namespace cmx {

// per-state flags
constexpr uint8_t SF_BEGL = 1;       // BEGL_S: deck is a ring of W+1 columns
constexpr uint8_t SF_TWO_SLOT = 2;   // right emitter: two column slots (j&1)
constexpr uint8_t SF_ENDSC = 4;      // endsc is possible: init_sc = el_sca[d]+endsc
constexpr uint8_t SF_BEGIN = 8;      // local-begin candidate (beginsc possible)

// Band + deck location of one state.  A read of cell d of state y returns
// deck[base(+slot*width) + d] when dn <= d <= dxcap, init0 when d == 0 and
// zero otherwise: exactly what the reference's full decks hold at those
// cells (never-written cells keep their IMPOSSIBLE / -INFTY fill).
struct alignas(16) StateDev {
    // first 16 bytes: everything a deck read needs (one vector load)
    int32_t base;     // deck offset of slot 0 minus dn
    int16_t dn;       // first d computed (>= 1)
    int16_t dxcap;    // min(dmax, W)
    int16_t width;    // dxcap - dn + 1 (0 when empty)
    uint8_t flags;    // SF_*
    uint8_t type;     // sttype
    int16_t cfirst;   // first child (B: BEGL state)
    int16_t cnum;     // children (B: BEGR state)
    // second 16 bytes
    int16_t kdn_y, kdx_y, kdn_w, kdx_w;  // B: raw clamped bands of BEGR / BEGL
    int32_t esc_off;  // row of the emission table (state index * 324)
    int32_t pad;
};
static_assert(sizeof(StateDev) == 32, "StateDev layout");

// A unit of work inside one level: state v, cells d0..d0+31 (warp-wide).
// For IL states d0 = -1: one warp resolves the whole band.
struct ChunkDev {
    int32_t v;
    int32_t d0;
};

struct Plan {
    int M = 0, W = 0;
    int semiring = 0, qdbidx = 0;
    std::vector<StateDev> states;
    std::vector<ChunkDev> chunks;
    std::vector<int32_t> level_start;   // nlev+1 offsets into chunks
    std::vector<int32_t> begin_states;  // local-begin candidates (ascending)
    int64_t deck_elems = 0;
    // score tables in the semiring's type, stored as 32-bit words
    std::vector<uint32_t> tsc;          // [M][6]
    std::vector<uint32_t> init0;        // [M] value of cell d = 0
    std::vector<uint32_t> endsc;        // [M]
    std::vector<uint32_t> beginsc;      // [M]
    std::vector<uint32_t> esc;          // [M][324]
    std::vector<uint32_t> el_sca;       // [W+1]
    int32_t root_dn = 0, root_dxcap = 0, root_cfirst = 0, root_cnum = 0;
    bool local = false;
    // exact work per column at full band (jrow = W): cells and child terms
    double cells_per_col = 0, terms_per_col = 0;
    int max_level_chunks = 0;
};

}  // namespace cmx
