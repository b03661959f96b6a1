/*
 * CPU oracle for the tree-layout hot path.  TEST INFRASTRUCTURE ONLY.
 *
 * This is a plain-C restatement of the reference algorithms (algoparc/Tree-Layouts)
 * for the in-place permutations sorted -> {level-order BST, level-order B-tree,
 * modified van Emde Boas} and for the point queries over those layouts.  Every
 * function cites the reference file:line it follows.  It exists so the tests,
 * the smoke check and the CPU-baseline leg of the benchmark can CHECK the CUDA
 * library; nothing in the shipped library links or calls it.
 *
 * Keys are handled as opaque 64-bit words for the permutations (they are pure
 * index permutations, oblivious to key values).  A 32-bit layout is the same
 * permutation: permute the identity 0..n-1 and apply it.
 *
 * Parity pins: B-tree and BST against the reference's own CPU code compiled from
 * its sources (oracle/Makefile -> oracle/_ref/libref_cpu.so); mvEB layout against
 * the reference's GPU code (oracle/_ref/libref_gpu.so) run on a B200, with the
 * outputs committed as fixtures under tests/golden/.
 */
#ifndef TL_ORACLE_H
#define TL_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Layout permutations, in place on n 64-bit words. Return 0 on success. */
int orc_permute_btree(uint64_t *A, uint64_t n, uint64_t b);
int orc_permute_bst(uint64_t *A, uint64_t n);
int orc_permute_mveb(uint64_t *A, uint64_t n);
/* the standard vEB of the reference's CPU code (cpu/src/veb-cycles.h) */
int orc_permute_veb_std(uint64_t *A, uint64_t n);

/* Point queries: ans[i] = position of q[i] in the layout, or n if absent.
 * Keys are compared as unsigned 64-bit integers (pass 32-bit keys widened). */
void orc_search_bst(const uint64_t *A, uint64_t n, const uint64_t *q, uint64_t nq, uint64_t *ans);
void orc_search_btree(const uint64_t *A, uint64_t n, uint64_t b, const uint64_t *q, uint64_t nq,
                      uint64_t *ans);

/* Brodal-Fagerberg-Jacob position table, same field order as the reference. */
typedef struct {
    uint64_t L; /* size of the bottom trees at this depth */
    uint64_t R; /* size of the corresponding top tree */
    uint32_t D; /* depth of the root of the corresponding top tree */
} orc_veb_table;

void orc_build_table(orc_veb_table *table, uint64_t n, uint32_t d, uint32_t root_depth);
/* Sizes of the non-perfect table set for n keys (num_tables, total entries). */
void orc_veb_tables_size(uint64_t n, uint32_t *num_tables, uint32_t *table_size);
/* Fills tables[table_size], idx[num_tables], table_idx[num_tables]. */
void orc_build_veb_tables(uint64_t n, orc_veb_table *tables, uint64_t *idx, uint32_t *table_idx);
void orc_build_table_std(orc_veb_table *table, uint64_t n, uint32_t d, uint32_t root_depth);
void orc_veb_tables_size_std(uint64_t n, uint32_t *num_tables, uint32_t *table_size);
void orc_build_veb_tables_std(uint64_t n, orc_veb_table *tables, uint64_t *idx, uint32_t *table_idx);
void orc_search_veb(const uint64_t *A, const orc_veb_table *table, uint64_t n, uint32_t d,
                    const uint64_t *q, uint64_t nq, uint64_t *ans);
void orc_search_veb_nonperfect(const uint64_t *A, const orc_veb_table *tables, const uint64_t *idx,
                               const uint32_t *table_idx, uint64_t n, uint32_t d,
                               uint32_t num_tables, const uint64_t *q, uint64_t nq,
                               uint64_t *ans);

/* Multithreaded timing helpers for the CPU baseline (OpenMP over queries). */
double orc_time_permute_btree(uint64_t *A, uint64_t n, uint64_t b);

#ifdef __cplusplus
}
#endif
#endif
