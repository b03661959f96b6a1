// Plan O tile order of the B-tree stream pass (btree_order.cu).
#pragma once

#include <vector>

#include "btree_plan.cuh"

namespace tl {

// The tables of plan O for one geometry (host or device pointers).
struct OrderTables {
    const uint2 *tab = nullptr;       // per tile {ticket, scratch slot or kNoSlot}
    const uint32_t *order = nullptr;  // tile of each ticket
    const uint32_t *list = nullptr;   // the tiles that receive scratch keys, ascending (slot order)
    uint64_t nlist = 0;
};

// Host vectors behind an OrderTables.
struct OrderVectors {
    std::vector<uint2> tab;
    std::vector<uint32_t> order, list;
    OrderTables tables() const {
        OrderTables t;
        t.tab = tab.data();
        t.order = order.data();
        t.list = list.data();
        t.nlist = list.size();
        return t;
    }
};

// Computes the tables for the geometry of S (S.plan and its tables are ignored).
void btree_compute_order(const BtreeStream &S, OrderVectors &v);

// Cached host tables for S's geometry; false when the cache is full.
bool btree_order_host(const BtreeStream &S, OrderTables &t);

// Cached device tables on the current device; false when they cannot be made
// now (the cache is full, the stream is being captured, or the copy failed).
bool btree_order_device(const BtreeStream &S, cudaStream_t st, OrderTables &t);

}  // namespace tl
