// Thin extern "C" shim over the reference's own CPU van Emde Boas code (TEST
// INFRASTRUCTURE): the standard vEB layout, its buildTable and its searches.
// Compiled by oracle/Makefile against the reference sources where they lie; the
// reference headers are included, never copied.  Output: oracle/_ref/libref_cpu.so.
#include "query-veb.h"   // cpu/src/query-veb.h: vEB_table, searchAll (:70-81), searchAll_nonperfect (:167-178)
#include "veb-cycles.h"  // cpu/src/veb-cycles.h: timePermutevEB (:380-395)

extern "C" double ref_cpu_permute_veb_u64(uint64_t *A, uint64_t n, uint32_t p) {
    return timePermutevEB<uint64_t>(A, n, p);
}
// cpu/src/query-veb.cpp:25-41
extern "C" void ref_cpu_build_table(vEB_table *table, uint64_t n, uint32_t d, uint32_t root_depth) {
    buildTable(table, n, d, root_depth);
}
// Hits only: on a miss the reference's descent writes pos[d], one past its array.
extern "C" void ref_cpu_search_veb_u64(uint64_t *A, vEB_table *table, uint64_t n, uint32_t d, uint64_t *q,
                                       uint64_t *ans, uint64_t nq, uint32_t p) {
    searchAll<uint64_t>(A, table, n, d, q, ans, nq, p);
}
// tables: num_tables pointers into one concatenated array (as the CPU driver
// allocates one table per division, cpu/test/query-veb-fixedN.cpp:116-150).
extern "C" void ref_cpu_search_veb_nonperfect_u64(uint64_t *A, vEB_table *concat, const uint32_t *table_idx,
                                                  uint64_t *idx, uint32_t num_tables, uint32_t d, uint64_t *q,
                                                  uint64_t *ans, uint64_t nq, uint32_t p) {
    vEB_table *tables[64];
    for (uint32_t i = 0; i < num_tables && i < 64; ++i) tables[i] = concat + table_idx[i];
    searchAll_nonperfect<uint64_t>(A, tables, idx, num_tables, d, q, ans, nq, p);
}
