// Thin extern "C" shim over the reference's own CPU BST code (TEST INFRASTRUCTURE).
// Compiled by oracle/Makefile against the reference sources where they lie.
#include "bst-involutions.h"  // cpu/src/bst-involutions.h: timePermuteBST (:119-144)
#include "query-bst.h"        // cpu/src/query-bst.h: searchAll (:45-51)

extern "C" double ref_cpu_permute_bst_u64(uint64_t *A, uint64_t n, uint32_t p) {
    return timePermuteBST<uint64_t>(A, n, p);
}
extern "C" void ref_cpu_search_bst_u64(uint64_t *A, uint64_t n, uint64_t *q, uint64_t *ans,
                                       uint64_t nq, uint32_t p) {
    searchAll<uint64_t>(A, n, q, ans, nq, p);
}
