/*
 * tree_layouts.h - C ABI of the B200 tree-layout library (libtreelayouts.so).
 *
 * In-place permutation of a sorted device array into an implicit search-tree
 * layout (level-order BST, level-order B-tree with b keys per node, modified van
 * Emde Boas), and batched exact point queries over those layouts.  Plain
 * pointers and sizes only; every call returns a tl_status.
 *
 * Each entry point names the reference (algoparc/Tree-Layouts) interface it
 * replaces.  The reference's C++ template names are re-exposed on top of this
 * ABI by tree_layouts.cuh.
 *
 * Conventions
 *  - dev_* pointers are device (HBM) pointers; host_* pointers are host memory.
 *  - stream: a cudaStream_t passed as void* (NULL = legacy default stream).
 *  - ms: if non-NULL the call synchronises the stream and stores the device time
 *    of the operation in milliseconds (CUDA events on `stream`).  Queries with
 *    ms == NULL are asynchronous with respect to the host.  Permutations always
 *    return after their work on `stream` has finished: they read back the status
 *    of their bounded device-side waits (TL_ERROR_TIMEOUT), like the reference's
 *    timePermute* functions, which end in cudaDeviceSynchronize.
 *  - Keys of a layout must be strictly increasing before a permutation for the
 *    queries to be meaningful; the permutations themselves move words and never
 *    look at key values.
 *  - Query answers are the layout position of the key, or n when absent (the
 *    reference's convention, gpu/src/query-bst.cuh:41).
 */
#ifndef TREE_LAYOUTS_H
#define TREE_LAYOUTS_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TL_VERSION 1

typedef enum tl_status {
    TL_SUCCESS = 0,
    TL_ERROR_INVALID_VALUE = 1,        /* null pointer, b == 0, unsupported key width */
    TL_ERROR_CUDA = 2,                 /* a CUDA runtime call failed */
    TL_ERROR_TIMEOUT = 3,              /* a bounded device-side wait gave up */
    TL_ERROR_OUT_OF_MEMORY = 4,        /* workspace allocation failed */
    TL_ERROR_WORKSPACE_TOO_SMALL = 5,  /* caller-supplied workspace below tl_permute_workspace_bytes */
    TL_ERROR_UNSUPPORTED = 6           /* size or parameter outside what this build handles */
} tl_status;

typedef enum tl_layout {
    TL_LAYOUT_BST = 0,
    TL_LAYOUT_BTREE = 1,
    TL_LAYOUT_MVEB = 2
} tl_layout;

/* Brodal-Fagerberg-Jacob position table; same layout (24 bytes) as the
 * reference's struct vEB_table, gpu/src/query-mveb.cuh:27-31. */
typedef struct tl_veb_table {
    uint64_t L; /* size of the bottom trees that start at this depth */
    uint64_t R; /* size of the corresponding top tree */
    uint32_t D; /* depth of the root of that top tree */
} tl_veb_table;

/* ---------------------------------------------------------------- misc */
int tl_version(void);
const char *tl_status_string(int status);
/* Last CUDA error seen by the library on this host thread (cudaError_t value). */
int tl_last_cuda_error(void);

/* Host-side layout geometry: position of sorted rank `rank` in the layout of n
 * keys (b ignored unless layout == TL_LAYOUT_BTREE). */
int tl_layout_position(int layout, uint64_t n, uint64_t b, uint64_t rank, uint64_t *pos);

/* ---------------------------------------------------------------- permutations */
/* Bytes of device workspace the permutation of (layout, n, b, key_bytes) uses. */
int tl_permute_workspace_bytes(int layout, uint64_t n, uint64_t b, uint32_t key_bytes,
                               uint64_t *bytes);

/* Generic in-place permutation sorted -> layout.  key_bytes is 4 or 8.
 * dev_workspace may be NULL: the library then allocates it stream-ordered
 * (cudaMallocAsync) and frees it before returning.
 * Replaces timePermuteBST (gpu/src/bst-involutions.cuh:168-195),
 * timePermuteBtree (gpu/src/btree-cycles.cuh:77-104) and
 * timePermutevEB (gpu/src/mveb-cycles.cuh:420-440). */
int tl_permute(int layout, void *dev_A, uint64_t n, uint64_t b, uint32_t key_bytes,
               void *dev_workspace, uint64_t workspace_bytes, void *stream, float *ms);

/* timePermuteBST<TYPE>(TYPE *dev_A, uint64_t n): gpu/src/bst-involutions.cuh:168 */
int tl_permute_bst_u32(uint32_t *dev_A, uint64_t n, void *stream, float *ms);
int tl_permute_bst_u64(uint64_t *dev_A, uint64_t n, void *stream, float *ms);
/* timePermuteBtree<TYPE>(TYPE *dev_A, uint64_t n, uint64_t b): gpu/src/btree-cycles.cuh:77 */
int tl_permute_btree_u32(uint32_t *dev_A, uint64_t n, uint64_t b, void *stream, float *ms);
int tl_permute_btree_u64(uint64_t *dev_A, uint64_t n, uint64_t b, void *stream, float *ms);
/* timePermutevEB<TYPE>(TYPE *dev_A, uint64_t n): gpu/src/mveb-cycles.cuh:420 */
int tl_permute_mveb_u32(uint32_t *dev_A, uint64_t n, void *stream, float *ms);
int tl_permute_mveb_u64(uint64_t *dev_A, uint64_t n, void *stream, float *ms);

/* No counterpart in the reference.  tl_permute for callers that cannot allocate
 * device memory (a plugin inside a host engine that owns every allocation, a
 * latency-bound service that must not hit cudaMalloc's implicit synchronisation
 * mid-request): the workspace is a fixed array of TL_STATIC_WORKSPACE_BYTES
 * compiled into the library, present on every GPU that loads it until the
 * process exits.  Permutations whose tl_permute_workspace_bytes exceeds it
 * return TL_ERROR_UNSUPPORTED.  All calls share that array: calls that overlap
 * on the GPU race, so serialise them.  The first call on a device looks the
 * array up (cudaGetSymbolAddress); make it before any stream capture.
 * Synchronous like tl_permute; allocates nothing. */
#define TL_STATIC_WORKSPACE_BYTES (32ull << 20)
int tl_permute_static_ws(int layout, void *dev_A, uint64_t n, uint64_t b, uint32_t key_bytes,
                         void *stream);

/* ---------------------------------------------------------------- mvEB tables */
/* buildTable(vEB_table *table, uint64_t n, uint32_t d, uint32_t root_depth):
 * gpu/src/query-mveb.cu:25-47.  Host function; table holds d entries, zeroed by
 * the caller as the reference's calloc does. */
void tl_build_table(tl_veb_table *table, uint64_t n, uint32_t d, uint32_t root_depth);
/* Sizes of the table set of a layout of n keys (one table when n = 2^d - 1):
 * the sizing loop of gpu/test/query-mveb-fixedN.cu:45-97.  d receives
 * log2(n) + 1. */
int tl_veb_tables_size(uint64_t n, uint32_t *num_tables, uint32_t *table_size, uint32_t *d);
/* Fills tables[table_size] (zeroed here), idx[num_tables], table_idx[num_tables]
 * exactly as gpu/test/query-mveb-fixedN.cu:130-165 builds them. */
int tl_build_veb_tables(uint64_t n, tl_veb_table *tables, uint64_t *idx, uint32_t *table_idx);

/* ---------------------------------------------------------------- queries */
/* dev_answers[i] = position of dev_queries[i] in the layout, or n.
 * searchAll (gpu/src/query-bst.cuh:47-54) behind timeQueryBST (:58-110). */
int tl_query_bst_u32(const uint32_t *dev_layout, uint64_t n, const uint32_t *dev_queries,
                     uint64_t q, uint64_t *dev_answers, void *stream, float *ms);
int tl_query_bst_u64(const uint64_t *dev_layout, uint64_t n, const uint64_t *dev_queries,
                     uint64_t q, uint64_t *dev_answers, void *stream, float *ms);
/* searchAll (gpu/src/query-btree.cuh:64-72) behind timeQueryBtree (:76-129); any
 * b >= 1 (the reference kernel assumes b = 32). */
int tl_query_btree_u32(const uint32_t *dev_layout, uint64_t n, uint64_t b,
                       const uint32_t *dev_queries, uint64_t q, uint64_t *dev_answers,
                       void *stream, float *ms);
int tl_query_btree_u64(const uint64_t *dev_layout, uint64_t n, uint64_t b,
                       const uint64_t *dev_queries, uint64_t q, uint64_t *dev_answers,
                       void *stream, float *ms);
/* searchAll (gpu/src/query-mveb.cuh:73-81) behind timeQueryvEB (:86-163). */
int tl_query_veb_u32(const uint32_t *dev_layout, const tl_veb_table *dev_table, uint64_t n,
                     uint32_t d, const uint32_t *dev_queries, uint64_t q, uint64_t *dev_answers,
                     void *stream, float *ms);
int tl_query_veb_u64(const uint64_t *dev_layout, const tl_veb_table *dev_table, uint64_t n,
                     uint32_t d, const uint64_t *dev_queries, uint64_t q, uint64_t *dev_answers,
                     void *stream, float *ms);
/* searchAll_nonperfect (gpu/src/query-mveb.cuh:218-226) behind
 * timeQueryvEB_nonperfect (:231-308). */
int tl_query_veb_nonperfect_u32(const uint32_t *dev_layout, const tl_veb_table *dev_tables,
                                const uint64_t *dev_idx, const uint32_t *dev_table_idx,
                                uint64_t n, uint32_t d, uint32_t num_tables,
                                const uint32_t *dev_queries, uint64_t q, uint64_t *dev_answers,
                                void *stream, float *ms);
int tl_query_veb_nonperfect_u64(const uint64_t *dev_layout, const tl_veb_table *dev_tables,
                                const uint64_t *dev_idx, const uint32_t *dev_table_idx,
                                uint64_t n, uint32_t d, uint32_t num_tables,
                                const uint64_t *dev_queries, uint64_t q, uint64_t *dev_answers,
                                void *stream, float *ms);

/* ---------------------------------------------------------------- test and profiling hooks */
/* Bound every device-side wait to spin_limit iterations (0 = default, about one
 * second) and, when force_timeout != 0, make the waits expect a flag value no
 * tile publishes, so they expire: exercises TL_ERROR_TIMEOUT without a fault. */
int tl_debug_set_wait(unsigned int spin_limit, int force_timeout);
/* Host replay of the permutation's tile schedule on a host array of n 64-bit
 * words, with the same index helpers as the kernels; *violations counts
 * protocol breaches (stale read, unguarded store, bad wait, position or scratch
 * slot not written exactly once). */
int tl_debug_emulate_permute(int layout, uint64_t n, uint64_t b, uint64_t *host_A, uint64_t *violations);
/* Schedule the B-tree permutation uses for (n, b): 0 right-to-left, 1 left-to-right. */
int tl_debug_btree_plan(uint64_t n, uint64_t b);
/* tl_permute with library-allocated workspace, reporting the device time of its
 * two passes: phase_ms[0] = setup + stream kernel, phase_ms[1] = scatter kernel. */
int tl_debug_permute_phases(int layout, void *dev_A, uint64_t n, uint64_t b, uint32_t key_bytes,
                            void *stream, float *phase_ms);

#ifdef __cplusplus
}
#endif
#endif
