/*
 * tree_layouts.cuh - the reference's C++ API (algoparc/Tree-Layouts, GPU side)
 * re-exposed as inline templates over the C ABI of libtreelayouts.so.
 *
 * A program written against the reference's gpu/src headers can include this
 * header instead and link -ltreelayouts:
 *
 *   timePermuteBST<TYPE>(dev_A, n)             gpu/src/bst-involutions.cuh:168
 *   timePermuteBtree<TYPE>(dev_A, n, b)        gpu/src/btree-cycles.cuh:77
 *   timePermutevEB<TYPE>(dev_A, n)             gpu/src/mveb-cycles.cuh:420
 *   timeQueryBST<TYPE>(A, dev_A, n, q)         gpu/src/query-bst.cuh:58
 *   timeQueryBtree<TYPE>(A, dev_A, n, b, q)    gpu/src/query-btree.cuh:76
 *   timeQueryvEB<TYPE>(A, dev_A, dev_table, n, d, q)                     gpu/src/query-mveb.cuh:86
 *   timeQueryvEB_nonperfect<TYPE>(A, dev_A, dev_tables, dev_idx, dev_table_idx, n, d, num_tables, q)
 *                                                                        gpu/src/query-mveb.cuh:231
 *   buildTable(table, n, d, root_depth) and struct vEB_table            gpu/src/query-mveb.cu:25
 *   timeQuery<TYPE>(A, dev_A, n, q)  (binary search, sorted dev_A)      gpu/src/binary-search.cuh:61
 *
 * Same argument meaning and return values: the permutations return host
 * wall-clock milliseconds including the final synchronisation; the queries
 * generate numQueries hit-only queries from A (as createRandomQueries does,
 * gpu/src/common.cuh:45-60, but from a fixed seed), copy A over dev_A, and
 * return the query kernel's device milliseconds.  Where the reference has no
 * error path these return a negative value on failure (see tl_status_string).
 * Permutations take any 4- or 8-byte TYPE; queries take unsigned 32/64-bit keys.
 */
#ifndef TREE_LAYOUTS_CUH
#define TREE_LAYOUTS_CUH

#include <cuda_runtime.h>
#include <stdint.h>
#include <stdlib.h>
#include <time.h>

#include <type_traits>
#include <vector>

#include "tree_layouts.h"

typedef tl_veb_table vEB_table;

namespace tree_layouts_api {

inline double wall_ms(const timespec &a, const timespec &b) {
    return ((b.tv_sec * 1e9 + b.tv_nsec) - (a.tv_sec * 1e9 + a.tv_nsec)) / 1e6;
}

template <typename TYPE>
inline double permute_timed(int layout, TYPE *dev_A, uint64_t n, uint64_t b) {
    static_assert(sizeof(TYPE) == 4 || sizeof(TYPE) == 8, "keys must be 4 or 8 bytes wide");
    timespec s, e;
    clock_gettime(CLOCK_MONOTONIC, &s);
    int rc = tl_permute(layout, dev_A, n, b, sizeof(TYPE), nullptr, 0, nullptr, nullptr);
    clock_gettime(CLOCK_MONOTONIC, &e);
    return rc == TL_SUCCESS ? wall_ms(s, e) : -1.0;
}

// Seed of the generated queries (the reference seeds rand() with time(NULL)).
inline uint64_t &query_seed() {
    static uint64_t seed = 0x5eed;
    return seed;
}

// splitmix64 (Steele, Lea, Flood, "Fast splittable pseudorandom number
// generators", OOPSLA 2014).
inline uint64_t splitmix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

// Hit-only queries drawn uniformly from the n keys in A.
template <typename TYPE>
inline std::vector<TYPE> random_queries(const TYPE *A, uint64_t n, uint64_t q) {
    std::vector<TYPE> out(q);
    const uint64_t seed = query_seed();
    for (uint64_t i = 0; i < q; ++i) out[i] = A[splitmix64(seed ^ (i * 0x2545F4914F6CDD1Dull)) % n];
    return out;
}

template <typename TYPE, typename Launch>
inline float query_timed(const TYPE *A, TYPE *dev_A, uint64_t n, uint64_t q, Launch launch) {
    static_assert(std::is_unsigned<TYPE>::value && (sizeof(TYPE) == 4 || sizeof(TYPE) == 8),
                  "queries compare unsigned 32- or 64-bit keys");
    std::vector<TYPE> queries = random_queries(A, n, q);
    TYPE *dev_q = nullptr;
    uint64_t *dev_ans = nullptr;
    if (cudaMalloc(&dev_q, q * sizeof(TYPE)) != cudaSuccess) return -1.f;
    if (cudaMalloc(&dev_ans, q * sizeof(uint64_t)) != cudaSuccess) {
        cudaFree(dev_q);
        return -1.f;
    }
    cudaMemcpy(dev_A, A, n * sizeof(TYPE), cudaMemcpyHostToDevice);
    cudaMemcpy(dev_q, queries.data(), q * sizeof(TYPE), cudaMemcpyHostToDevice);
    float ms = 0.f;
    int rc = launch(dev_q, dev_ans, &ms);
    cudaFree(dev_q);
    cudaFree(dev_ans);
    return rc == TL_SUCCESS ? ms : -1.f;
}

}  // namespace tree_layouts_api

template <typename TYPE>
inline float timePermuteBST(TYPE *dev_A, uint64_t n) {
    return (float)tree_layouts_api::permute_timed(TL_LAYOUT_BST, dev_A, n, 1);
}

template <typename TYPE>
inline double timePermuteBtree(TYPE *dev_A, uint64_t n, uint64_t b) {
    return tree_layouts_api::permute_timed(TL_LAYOUT_BTREE, dev_A, n, b);
}

template <typename TYPE>
inline double timePermutevEB(TYPE *dev_A, uint64_t n) {
    return tree_layouts_api::permute_timed(TL_LAYOUT_MVEB, dev_A, n, 0);
}

inline void buildTable(vEB_table *table, uint64_t n, uint32_t d, uint32_t root_depth) {
    tl_build_table(table, n, d, root_depth);
}

template <typename TYPE>
inline float timeQuery(TYPE *A, TYPE *dev_A, uint64_t n, uint64_t numQueries) {
    return tree_layouts_api::query_timed(A, dev_A, n, numQueries, [&](TYPE *q, uint64_t *ans, float *ms) {
        if (sizeof(TYPE) == 8)
            return tl_query_sorted_u64((const uint64_t *)dev_A, n, (const uint64_t *)q, numQueries, ans, nullptr,
                                       ms);
        return tl_query_sorted_u32((const uint32_t *)dev_A, n, (const uint32_t *)q, numQueries, ans, nullptr, ms);
    });
}

template <typename TYPE>
inline float timeQueryBST(TYPE *A, TYPE *dev_A, uint64_t n, uint64_t numQueries) {
    return tree_layouts_api::query_timed(A, dev_A, n, numQueries, [&](TYPE *q, uint64_t *ans, float *ms) {
        if (sizeof(TYPE) == 8)
            return tl_query_bst_u64((const uint64_t *)dev_A, n, (const uint64_t *)q, numQueries, ans, nullptr, ms);
        return tl_query_bst_u32((const uint32_t *)dev_A, n, (const uint32_t *)q, numQueries, ans, nullptr, ms);
    });
}

template <typename TYPE>
inline float timeQueryBtree(TYPE *A, TYPE *dev_A, uint64_t n, uint64_t b, uint64_t numQueries) {
    return tree_layouts_api::query_timed(A, dev_A, n, numQueries, [&](TYPE *q, uint64_t *ans, float *ms) {
        if (sizeof(TYPE) == 8)
            return tl_query_btree_u64((const uint64_t *)dev_A, n, b, (const uint64_t *)q, numQueries, ans, nullptr,
                                      ms);
        return tl_query_btree_u32((const uint32_t *)dev_A, n, b, (const uint32_t *)q, numQueries, ans, nullptr, ms);
    });
}

template <typename TYPE>
inline float timeQueryvEB(TYPE *A, TYPE *dev_A, vEB_table *dev_table, uint64_t n, uint32_t d, uint64_t numQueries) {
    return tree_layouts_api::query_timed(A, dev_A, n, numQueries, [&](TYPE *q, uint64_t *ans, float *ms) {
        if (sizeof(TYPE) == 8)
            return tl_query_veb_u64((const uint64_t *)dev_A, dev_table, n, d, (const uint64_t *)q, numQueries, ans,
                                    nullptr, ms);
        return tl_query_veb_u32((const uint32_t *)dev_A, dev_table, n, d, (const uint32_t *)q, numQueries, ans,
                                nullptr, ms);
    });
}

template <typename TYPE>
inline float timeQueryvEB_nonperfect(TYPE *A, TYPE *dev_A, vEB_table *dev_tables, uint64_t *dev_idx,
                                     uint32_t *dev_table_idx, uint64_t n, uint32_t d, uint32_t num_tables,
                                     uint64_t numQueries) {
    return tree_layouts_api::query_timed(A, dev_A, n, numQueries, [&](TYPE *q, uint64_t *ans, float *ms) {
        if (sizeof(TYPE) == 8)
            return tl_query_veb_nonperfect_u64((const uint64_t *)dev_A, dev_tables, dev_idx, dev_table_idx, n, d,
                                               num_tables, (const uint64_t *)q, numQueries, ans, nullptr, ms);
        return tl_query_veb_nonperfect_u32((const uint32_t *)dev_A, dev_tables, dev_idx, dev_table_idx, n, d,
                                           num_tables, (const uint32_t *)q, numQueries, ans, nullptr, ms);
    });
}

#endif
