// Plan of the node-sweep scan kernel (sweep_scan.cu): the CM's nodes in
// sweep order, per-state cell ranges and child locations, and the states
// whose previous-column values the next column needs.
//
// The kernel relies on the node-local topology every CM built by
// cm_from_guide has (src/cm_modelmaker.rs:979-1110): the children of a
// state of node n are node n's own insert states followed by the split
// states (the non-insert states) of node n+1; a bifurcation's children are
// the BEGL_S and BEGR_S states that start its two subtrees.  The builder
// checks this for every state and declines models that do not follow it.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/cmscan_gpu.h"
#include "qdb_plan.h"

namespace cmx {

constexpr int SW_SLOTS = 6;          // state slots of one node buffer
constexpr int SW_MAX_S = 256;        // words per slot: the kernel takes W <= 255

// Per-state metadata (16 bytes).
struct SwState {
    int16_t lo, hi;      // cells written every column: own band plus every index a reader uses
    int16_t dn, dxcap;   // band (as generic_scan's dn_v / dxcap_v)
    uint8_t type;        // sttype
    uint8_t flags;       // SF_* of qdb_plan.h, plus SWF_* below
    uint8_t cnum;        // children (B: 2)
    uint8_t sd;          // state delta
    int16_t escoff;      // row of the compact emission table (-1: none)
    uint8_t slot;        // slot in its node's buffer
    uint8_t pad;
};
static_assert(sizeof(SwState) == 16, "SwState layout");

constexpr uint8_t SWF_ROOT = 0x20;   // ROOT_S: plain child order, local begins, reporting
constexpr uint8_t SWF_BEGR = 0x40;   // BEGR_S: values go to the bifurcation's BEGR row
constexpr uint8_t SWF_BEGL = 0x80;   // BEGL_S: values go to the bifurcation's BEGL ring

// Where a child's value of the current column is read from (one byte per
// child): kind * 8 + slot, kind 0 = own node buffer, 1 = next node's buffer,
// 2 = the previous-column buffer of the node.
constexpr uint8_t KID_OWN = 0, KID_NEXT = 1, KID_PREV = 2;

// One node in sweep order (16 bytes).
struct SwNode {
    uint8_t type, nst;   // node type (cm_internal.h *_ND), number of states
    uint8_t nio;         // states whose previous-column values the node reads
    uint8_t aux;         // BIF / BEGL / BEGR: index of the bifurcation
    int16_t v0;          // first state
    int16_t io0;         // first entry of the node in the io list
    int32_t pad0, pad1;
};
static_assert(sizeof(SwNode) == 16, "SwNode layout");

// A state whose previous-column values node n reads (its own inserts, or
// the split states of node n+1): loaded from the warp's deck slot into the
// previous-column buffer before the node runs, and its current values
// stored to the deck slot after the node ran (16 bytes).
struct SwIO {
    int16_t y;           // state
    uint8_t pslot;       // slot in the previous-column buffer
    uint8_t cur;         // current values: 0..5 own buffer slot, 8+s next node's slot s
    int16_t lo, hi;      // cells
    int32_t deck;        // word offset of the deck slot
    int32_t pad;
};
static_assert(sizeof(SwIO) == 16, "SwIO layout");

// A bifurcation: the k-range clamps of generic_scan (src/cm_nohmm.rs:578-600).
struct SwBif {
    int16_t kdn_y, kdx_y, kdn_w, kdx_w;  // BEGR (y) and BEGL (w) d-ranges, capped at W
    int16_t begl, begr;                  // BEGL_S and BEGR_S states
    int16_t b, pad;                      // B state
};
static_assert(sizeof(SwBif) == 16, "SwBif layout");

struct SweepPlan {
    int M = 0, W = 0, S = 0, RW = 0;     // S: words per slot; RW: columns of a BEGL ring
    std::vector<SwState> st;
    std::vector<uint8_t> kid;            // [M][6]
    std::vector<SwNode> nodes;           // nodes[n] is node n; the sweep runs n descending
    std::vector<SwIO> io;
    std::vector<SwBif> bifs;
    int64_t deck_words = 0;              // per warp: previous-column deck slots
    int64_t ring_words = 0;              // per warp: BEGL rings (nbif * RW * S)
};

// Builds the sweep plan from the scan plan of the same (semiring, band set).
// Returns false (with the reason) when the model's topology or W is outside
// what the kernel handles; the caller then uses the level-scheduled kernel.
bool build_sweep_plan(const cmgpu_cm *cm, const Plan &p, int qdbidx, SweepPlan &sp, std::string *why);

}  // namespace cmx
