// Plan O tile order of the B-tree stream pass (btree_order.cu).
#pragma once

#include <vector>

#include "btree_plan.cuh"

namespace tl {

// A copy of the fix pass: len keys from scratch index src on to position dst
// on; dst in the low 48 bits of dst_len, len (at most kFixSegMax) in the high 16.
struct FixSeg {
    uint64_t dst_len, src;
};
constexpr uint64_t kFixSegMax = 8192;
constexpr uint64_t kSegDstMask = (1ull << 48) - 1;

// The tables of plan O for one geometry (tab, order and segs: host or device
// pointers; ranges: host).  The tiles that receive scratch keys own a tile of
// scratch each, in ascending order; runs of consecutive tiles whose every key
// goes through scratch are copied back as ranges by the bulk-copy engine (at
// most kMaxBulkRanges of them, the longest), the scratch keys of the other
// tiles by the fix pass, as the host-listed copies segs.
struct OrderTables {
    const uint2 *tab = nullptr;       // per tile {ticket, scratch slot or kNoSlot}
    const uint32_t *order = nullptr;  // tile of each ticket
    const FixSeg *segs = nullptr;     // the fix pass's copies
    uint64_t nsegs = 0;
    const uint4 *ranges = nullptr;    // tiles [x, y) from scratch slot z on, for the bulk-copy engine
    uint64_t nranges = 0;
    uint64_t scratch_tiles = 0;
};

// Host vectors behind an OrderTables.
struct OrderVectors {
    std::vector<uint2> tab;
    std::vector<uint4> ranges;
    std::vector<uint32_t> order;
    std::vector<FixSeg> segs;
    uint64_t scratch_tiles = 0;
    OrderTables tables() const {
        OrderTables t;
        t.tab = tab.data();
        t.order = order.data();
        t.segs = segs.data();
        t.nsegs = segs.size();
        t.ranges = ranges.data();
        t.nranges = ranges.size();
        t.scratch_tiles = scratch_tiles;
        return t;
    }
};

// Computes the tables for the geometry of S (S.plan and its tables are ignored).
void btree_compute_order(const BtreeStream &S, OrderVectors &v);

// The same tables with their two per-tile passes (pred, and the scratch counts
// under both tie orders) as kernels on st; the chain walk, the tickets and the
// rest on the host.  False on any CUDA failure (v then undefined).
bool btree_compute_order_device(const BtreeStream &S, cudaStream_t st, OrderVectors &v);

// Computes and caches S's tables with kernels on st (their two per-tile passes)
// when they are not cached yet; false if that cannot be done (the cache is
// full, st is being captured, a CUDA call failed): btree_order_host then
// computes them on the host.
bool btree_order_prepare(const BtreeStream &S, cudaStream_t st);

// Cached host tables for S's geometry; false when the cache is full.
bool btree_order_host(const BtreeStream &S, OrderTables &t);

// Cached device tables on the current device; false when they cannot be made
// now (the cache is full, the stream is being captured, or the copy failed).
bool btree_order_device(const BtreeStream &S, cudaStream_t st, OrderTables &t);

}  // namespace tl
