// Thin extern "C" shim over the reference's own CPU B-tree code (TEST INFRASTRUCTURE).
// Compiled by oracle/Makefile against the reference sources where they lie; the
// reference headers are included, never copied.  Output: oracle/_ref/libref_cpu.so.
#include "btree-cycles.h"  // cpu/src/btree-cycles.h: timePermuteBtree (:71-96)
#include "query-btree.h"   // cpu/src/query-btree.h: searchAll (:58-64)

extern "C" double ref_cpu_permute_btree_u64(uint64_t *A, uint64_t n, uint64_t b, uint32_t p) {
    return timePermuteBtree<uint64_t>(A, n, b, p);
}
extern "C" double ref_cpu_permute_btree_u32(uint32_t *A, uint64_t n, uint64_t b, uint32_t p) {
    return timePermuteBtree<uint32_t>(A, n, b, p);
}
// A must hold b padding words (UINT64_MAX) past n: the reference's node scan
// reads past the last, partially filled node (cpu/src/query-btree.h:40-41).
extern "C" void ref_cpu_search_btree_u64(uint64_t *A, uint64_t n, uint64_t b, uint64_t *q,
                                         uint64_t *ans, uint64_t nq, uint32_t p) {
    searchAll<uint64_t>(A, n, b, q, ans, nq, p);
}
