// Cooperative B-tree descent for the query kernels (sm_100a).
//
// A node of b keys is read by a group of G lanes, KPL keys each (G * KPL >= b;
// one 16-byte load per lane for b * w = 16 * G on an aligned layout): a warp
// instruction then touches 32 / G node lines instead of 32, and the query is
// ranked against the node with warp ballots (lane j of the group holds node
// slots [j * KPL, (j + 1) * KPL)).
// Each group keeps QK descents in flight; a slot whose descent ends writes its
// answer and takes the next query from a warp-wide queue of prepared queries
// (32 at a time, one per lane: the query key is read coalesced and, for the
// learned-start query, the rank model runs there, lane-parallel).  The warp
// leaves the loop when its range of queries is exhausted and every slot idle.
//
// The descent rule is the reference's searchBtree (cpu/src/query-btree.h:33-54,
// gpu/src/query-btree.cuh:32-62): follow the child numbered by the count of
// node keys smaller than the query, child of node i = (i + 1)(b + 1) + lt b - 1;
// an equal key ends the search at its position; falling off the tree answers n.
// Node slots at or past n (the partial last leaf) count as absent.
//
// The first P keys of the layout (whole top levels) may be pinned in shared
// memory; a node starting below P is read from there.
#pragma once

#include "tl_common.cuh"

namespace tl {

constexpr uint64_t kSlotIdle = ~0ull;

// A prepared query: key (zero-extended), start node, policy flags; `valid`
// false past the end of the warp's range.
struct QEntry {
    uint64_t key;
    uint64_t node;
    uint32_t flags;
    bool valid;
};

template <typename K>
__device__ __forceinline__ K key_from(uint64_t v) {
    return (K)v;
}

// Lowest `count` set bits of mask.
__device__ __forceinline__ unsigned lowest_bits(unsigned mask, uint32_t count) {
    unsigned take = 0;
    for (uint32_t c = 0; c < count && mask; ++c) {
        const unsigned low = mask & (0u - mask);
        take |= low;
        mask ^= low;
    }
    return take;
}

// The node row of lane gl of its group: node slots [gl * KPL, (gl + 1) * KPL)
// and how many of them hold keys (slots at or past b or past n hold none).
template <typename K, int KPL>
struct NodeRow {
    K k[KPL];
    uint32_t valid;
};

// Vector rows (one 8- or 16-byte load) need KPL * w in {8, 16} and node starts
// aligned to it: b * w a multiple of KPL * w and an aligned layout base.
template <typename K, int KPL>
constexpr bool kVecRow = KPL > 1 && (KPL * sizeof(K) == 16 || KPL * sizeof(K) == 8);

template <typename K, int KPL>
__device__ __forceinline__ void load_slots(const K *src, NodeRow<K, KPL> &row) {
    if constexpr (kVecRow<K, KPL> && KPL * sizeof(K) == 16) {
        const uint4 v = *reinterpret_cast<const uint4 *>(src);
        const K *kk = reinterpret_cast<const K *>(&v);
#pragma unroll
        for (int e = 0; e < KPL; ++e) row.k[e] = kk[e];
    } else if constexpr (kVecRow<K, KPL>) {
        const uint2 v = *reinterpret_cast<const uint2 *>(src);
        const K *kk = reinterpret_cast<const K *>(&v);
#pragma unroll
        for (int e = 0; e < KPL; ++e) row.k[e] = kk[e];
    } else {
#pragma unroll
        for (int e = 0; e < KPL; ++e) row.k[e] = src[e];
    }
}

template <typename K, int KPL>
__device__ __forceinline__ void load_slots_ldg(const K *__restrict__ src, NodeRow<K, KPL> &row) {
    if constexpr (kVecRow<K, KPL> && KPL * sizeof(K) == 16) {
        const uint4 v = __ldg(reinterpret_cast<const uint4 *>(src));
        const K *kk = reinterpret_cast<const K *>(&v);
#pragma unroll
        for (int e = 0; e < KPL; ++e) row.k[e] = kk[e];
    } else if constexpr (kVecRow<K, KPL>) {
        const uint2 v = __ldg(reinterpret_cast<const uint2 *>(src));
        const K *kk = reinterpret_cast<const K *>(&v);
#pragma unroll
        for (int e = 0; e < KPL; ++e) row.k[e] = kk[e];
    } else {
#pragma unroll
        for (int e = 0; e < KPL; ++e) row.k[e] = __ldg(src + e);
    }
}

template <typename K, int KPL>
__device__ __forceinline__ void load_row(const K *__restrict__ A, const K *sm, uint64_t P, uint64_t n, uint64_t b,
                                         uint64_t node, uint32_t gl, bool active, NodeRow<K, KPL> &row) {
    row.valid = 0;
#pragma unroll
    for (int e = 0; e < KPL; ++e) row.k[e] = K(0);
    if (!active) return;
    const uint64_t lim = n - node < b ? n - node : b;  // keys in this node
    const uint64_t j0 = (uint64_t)gl * KPL;
    if (j0 + KPL <= lim) {
        if (node < P)
            load_slots<K, KPL>(sm + node + j0, row);
        else
            load_slots_ldg<K, KPL>(A + node + j0, row);
        row.valid = KPL;
    } else if (j0 < lim) {  // the row that ends the node (b not a multiple of KPL, or the partial last leaf)
        row.valid = (uint32_t)(lim - j0);
#pragma unroll
        for (int e = 0; e < KPL; ++e)
            if ((uint32_t)e < row.valid) row.k[e] = node < P ? sm[node + j0 + e] : __ldg(A + node + j0 + e);
    }
}

// Rank of q in the group's node: lt = node keys < q, eq = some node key == q.
// Every lane of the warp must call it (ballots).
template <typename K, int KPL>
__device__ __forceinline__ void rank_row(const NodeRow<K, KPL> &row, K q, unsigned gmask, uint32_t &lt, bool &eq) {
    lt = 0;
    bool e_any = false;
#pragma unroll
    for (int e = 0; e < KPL; ++e) {
        const bool v = (uint32_t)e < row.valid;
        lt += __popc(__ballot_sync(0xFFFFFFFFu, v && row.k[e] < q) & gmask);
        e_any |= v && row.k[e] == q;
    }
    eq = (__ballot_sync(0xFFFFFFFFu, e_any) & gmask) != 0;
}

// Policy hooks (see PlainPolicy): prepare(Q, qi, valid) -> QEntry, one query
// per lane; seen(flags, lt, cnt) accumulates what a descent saw at a node of
// cnt keys; fell_off(node, flags, leader) -> true to answer n, false to go on
// from the node it writes (a restart); answer(ans, qi, res) stores a result.
// seen and fell_off run in every lane of the slot's group; `leader` is true in
// one of them; answer runs in the leader only.
struct PlainPolicy {
    template <typename K>
    __device__ __forceinline__ QEntry prepare(const K *__restrict__ Q, uint64_t qi, bool valid) const {
        QEntry e;
        e.key = valid ? (uint64_t)__ldcs(Q + qi) : 0;
        e.node = 0;
        e.flags = 0;
        e.valid = valid;
        return e;
    }
    __device__ __forceinline__ uint32_t seen(uint32_t flags, uint32_t, uint32_t) const { return flags; }
    __device__ __forceinline__ bool fell_off(uint64_t &, uint32_t &, bool) { return true; }
    __device__ __forceinline__ void answer(uint64_t *__restrict__ ans, uint64_t qi, uint64_t res) const {
        __stcs(ans + qi, res);
    }
};

// One warp answers queries [q0, q1) of Q into ans: G lanes per node, KPL node
// slots per lane (G * KPL >= b), QK descents in flight per group.
template <typename K, int G, int KPL, int QK, typename Policy>
__device__ __forceinline__ void btree_descend_warp(const K *__restrict__ A, const K *sm, uint64_t P, uint64_t n,
                                                   uint64_t b, const K *__restrict__ Q, uint64_t q0, uint64_t q1,
                                                   uint64_t *__restrict__ ans, Policy &pol) {
    static_assert(G >= 1 && G <= 32 && (G & (G - 1)) == 0, "G: a power of two up to 32");
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t gl = lane & (G - 1);
    const uint32_t gbase = lane - gl;
    const unsigned gmask = (G == 32 ? 0xFFFFFFFFu : ((1u << G) - 1u)) << gbase;
    const unsigned lt_leader = (1u << gbase) - 1u;  // lanes below this group's leader
    const uint64_t cmax = (n + 1) / (b + 1);

    uint64_t node[QK], qid[QK];
    K qk[QK];
    uint32_t fl[QK];
#pragma unroll
    for (int k = 0; k < QK; ++k) {
        node[k] = kSlotIdle;
        qid[k] = 0;
        qk[k] = K(0);
        fl[k] = 0;
    }
    // prepared queue: lane l holds entry l of the current batch
    QEntry ent;
    ent.valid = false;
    uint64_t next = q0, batch0 = q0;
    uint32_t bn = 0, bpos = 0;

    for (;;) {
        // refill idle slots from the queue
#pragma unroll
        for (int k = 0; k < QK; ++k) {
            unsigned need = __ballot_sync(0xFFFFFFFFu, node[k] == kSlotIdle && gl == 0);
            while (need) {
                if (bpos == bn) {
                    if (next >= q1) break;
                    batch0 = next;
                    bn = (uint32_t)(q1 - next < 32 ? q1 - next : 32);
                    bpos = 0;
                    next += bn;
                    ent = pol.prepare(Q, batch0 + lane, lane < bn);
                }
                const unsigned take = lowest_bits(need, bn - bpos);
                const bool mine = (take >> gbase) & 1u;
                const uint32_t src = bpos + __popc(take & lt_leader);
                const uint64_t key = __shfl_sync(0xFFFFFFFFu, ent.key, mine ? src : 0);
                const uint64_t nd = __shfl_sync(0xFFFFFFFFu, ent.node, mine ? src : 0);
                const uint32_t f = __shfl_sync(0xFFFFFFFFu, ent.flags, mine ? src : 0);
                if (mine) {
                    qk[k] = key_from<K>(key);
                    node[k] = nd;
                    fl[k] = f;
                    qid[k] = batch0 + src;
                }
                bpos += __popc(take);
                need &= ~take;
            }
        }
        bool busy = false;
#pragma unroll
        for (int k = 0; k < QK; ++k) busy |= node[k] != kSlotIdle;
        if (!__any_sync(0xFFFFFFFFu, busy)) break;

        // one level of every busy slot: all loads first, then the ranks
        NodeRow<K, KPL> row[QK];
#pragma unroll
        for (int k = 0; k < QK; ++k) load_row<K, KPL>(A, sm, P, n, b, node[k], gl, node[k] != kSlotIdle, row[k]);
#pragma unroll
        for (int k = 0; k < QK; ++k) {
            uint32_t lt;
            bool eq;
            rank_row<K, KPL>(row[k], qk[k], gmask, lt, eq);
            if (node[k] == kSlotIdle) continue;
            uint64_t res = kSlotIdle;
            if (eq) {
                res = node[k] + lt;
            } else {
                fl[k] = pol.seen(fl[k], lt, (uint32_t)(n - node[k] < b ? n - node[k] : b));
                uint64_t nx = n;
                if (node[k] + 1 <= cmax) nx = (node[k] + 1) * (b + 1) + (uint64_t)lt * b - 1;
                if (nx < n) {
                    node[k] = nx;
                } else if (pol.fell_off(node[k], fl[k], gl == 0)) {
                    res = n;
                }
            }
            if (res != kSlotIdle) {
                if (gl == 0) pol.answer(ans, qid[k], res);
                node[k] = kSlotIdle;
            }
        }
    }
}

}  // namespace tl
