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

// Deck layout.  Every state y owns `slots` column slots of `span` cells,
// covering indices lo..hi: its own band [dn, dxcap] and every index any
// parent, the root or a bifurcation reads (d - sd of the parent's band).
// Cells outside the band are never written, so they keep the fill the
// reference's full decks hold there: the d = 0 base value at index 0 and
// IMPOSSIBLE / -INFTY elsewhere.  A child read is then one load at
// cb[v][yo][j & 1] + d, with no range test.
struct StateDev {
    int16_t dn;       // first d computed (>= 1)
    int16_t dxcap;    // min(dmax, W)
    uint8_t cnum;     // children (B: 2)
    uint8_t type;     // sttype
    uint8_t flags;    // SF_*
    uint8_t sd;       // state delta (residues emitted)
    int32_t escoff;   // row of the compact emission table (-1: none)
    int32_t span;     // cells per deck slot (0: no deck)
};
static_assert(sizeof(StateDev) == 16, "StateDev layout");

// A unit of work inside one level: state v, cells d0..d0+63 (a warp, two
// cells per lane).
// For IL states d0 = -1: one warp resolves the whole band.
struct ChunkDev {
    int32_t v;
    int32_t d0;
};

// A local-begin candidate of the ROOT_S reduction.
struct BeginDev {
    int32_t v;
    int32_t base0, base1;  // deck base of column parity 0 / 1 (BEGL: ring slot 0)
    int16_t dn, dxcap;
};
static_assert(sizeof(BeginDev) == 16, "BeginDev layout");

struct Plan {
    int M = 0, W = 0;
    int semiring = 0, qdbidx = 0;
    std::vector<StateDev> states;
    std::vector<int32_t> wb;            // [M][2] own write base by column parity
    std::vector<int32_t> cb;            // [M][12]: child yo, column parity par at
                                        // [2*yo+par], read base minus sd.  B states:
                                        // [0..1] BEGL ring base, [2..3] BEGR base,
                                        // [4..7] kdn_y kdx_y kdn_w kdx_w, [8] BEGL span
    std::vector<ChunkDev> chunks;
    std::vector<int32_t> level_start;   // nlev+1 offsets into chunks
    std::vector<BeginDev> begins;       // local-begin candidates (ascending v)
    std::vector<uint32_t> beginsc;      // score of each begin candidate
    std::vector<int32_t> init_off;      // deck cells holding a d = 0 base value
    std::vector<uint32_t> init_val;
    int64_t deck_elems = 0;
    // score tables in the semiring's type, stored as 32-bit words
    std::vector<uint32_t> tsc;          // [M][6]
    std::vector<uint32_t> init0;        // [M] value of cell d = 0
    std::vector<uint32_t> endsc;        // [M]
    std::vector<uint32_t> beginsc_all;  // [M]
    std::vector<uint32_t> esc;          // [M][324]
    std::vector<int32_t> escoff;        // [M] offset into esc_c (-1: no emission)
    std::vector<uint32_t> esc_c;        // canonical emissions: 4 per single, 16 per pair
    std::vector<uint32_t> el_sca;       // [W+1]
    int32_t root_dn = 0, root_dxcap = 0, root_cnum = 0;
    bool local = false;
    int max_level_chunks = 0;
};

}  // namespace cmx
