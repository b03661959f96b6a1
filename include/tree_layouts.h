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
    TL_LAYOUT_MVEB = 2,
    TL_LAYOUT_VEB = 3  /* the standard van Emde Boas layout of the reference's CPU code */
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
/* Bytes of device workspace the permutation of (layout, n, b, key_bytes) may
 * use: enough for the ordered-tile schedule and for the fixed-direction one it
 * falls back to, so a workspace of this size is always accepted. */
int tl_permute_workspace_bytes(int layout, uint64_t n, uint64_t b, uint32_t key_bytes,
                               uint64_t *bytes);

/* Generic in-place permutation sorted -> layout.  key_bytes is 4 or 8.
 * dev_workspace may be NULL: the library then takes a device buffer from a
 * small per-device cache that it fills with cudaMalloc (at most 8 buffers,
 * kept for the life of the process, each lent to one call at a time; when no
 * cached buffer can be had, a stream-ordered cudaMallocAsync that the call
 * frees before returning).
 * Per-geometry tables: a B-tree or BST of 64 tiles or more (16384 for the BST)
 * takes the ordered-tile schedule, whose tables depend only on (n, b, tile
 * size).  The first call for a new geometry on a device builds them and copies
 * them into a cudaMalloc'd block that the library keeps for the life of the
 * process (at most 64 geometries, about 12 bytes per 32 KB tile plus the fix
 * segments); that first call therefore allocates and synchronises even when
 * dev_workspace is given.  If the tables cannot be built or copied (out of
 * memory, a capturing stream, more than 64 devices or geometries) the call
 * takes the fixed-direction schedule instead, which the workspace size above
 * covers.
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
/* The standard van Emde Boas layout (root floor(d/2), bottoms ceil(d/2) levels),
 * which the reference builds on the CPU only: timePermutevEB<TYPE>(TYPE *A,
 * uint64_t n, uint32_t p), cpu/src/veb-cycles.h:380-395.  Here on the device,
 * in place, as tl_permute(TL_LAYOUT_VEB, ...). */
int tl_permute_veb_std_u32(uint32_t *dev_A, uint64_t n, void *stream, float *ms);
int tl_permute_veb_std_u64(uint64_t *dev_A, uint64_t n, void *stream, float *ms);

/* No counterpart in the reference.  tl_permute for callers that cannot allocate
 * device memory (a plugin inside a host engine that owns every allocation, a
 * latency-bound service that must not hit cudaMalloc's implicit synchronisation
 * mid-request): the workspace is a fixed array of TL_STATIC_WORKSPACE_BYTES
 * compiled into the library, present on every GPU that loads it until the
 * process exits.  It keeps to the fixed-direction schedules (the ordered one
 * needs per-size tables the library would allocate); permutations whose
 * workspace under those exceeds the array return TL_ERROR_UNSUPPORTED.  All
 * calls share that array: calls that overlap on the GPU race, so serialise
 * them.  The first call on a device looks the array up (cudaGetSymbolAddress);
 * make it before any stream capture.  Synchronous like tl_permute: it reads
 * back the status of its device waits and returns after its work on `stream`
 * has finished.  Allocates nothing. */
#define TL_STATIC_WORKSPACE_BYTES (32ull << 20)
int tl_permute_static_ws(int layout, void *dev_A, uint64_t n, uint64_t b, uint32_t key_bytes,
                         void *stream);

/* The reference's algorithm families as variants of tl_permute (its library
 * ships several for each layout: cycle-leader, involutions, hybrid), for
 * ablations and as other routes to the same layout:
 *  - TL_ALGO_STREAM: this library's own single-pass stream permutation (what
 *    tl_permute runs);
 *  - TL_ALGO_INVOLUTIONS: the BST, the B-tree or the mvEB by involutions
 *    (gpu/src/bst-involutions.cuh:168-195 timePermuteBST,
 *    gpu/src/btree-involutions.cuh:148-168 timePermuteBtree, b 1 .. 2^31 - 1;
 *    gpu/src/mveb-involutions.cuh:502-523 timePermutevEB);
 *  - TL_ALGO_CYCLES: the B-tree (b 1 .. 2^20 - 1), the BST (the B-tree with
 *    b = 1) or the mvEB by the cycle-leader family, equidistant gathers and
 *    rotations (gpu/src/btree-cycles.cuh:77-104 timePermuteBtree,
 *    gpu/test/build-bst-cycles.cu:39, gpu/src/mveb-cycles.cuh:420-440
 *    timePermutevEB);
 *  - TL_ALGO_HYBRID: the BST's last level by cycles and its perfect part by
 *    involutions (gpu/src/bst-hybrid.cuh:121-148 timePermuteBST).
 * Other (layout, algorithm) pairs return TL_ERROR_UNSUPPORTED.  Allocates
 * nothing beyond what tl_permute does; synchronous; ms as for tl_permute. */
typedef enum { TL_ALGO_STREAM = 0, TL_ALGO_INVOLUTIONS = 1, TL_ALGO_CYCLES = 2, TL_ALGO_HYBRID = 3 } tl_algorithm;
int tl_permute_algorithm(int layout, int algorithm, void *dev_A, uint64_t n, uint64_t b, uint32_t key_bytes,
                         void *stream, float *ms);

/* The reverse permutation: a layout of n sorted keys (as tl_permute leaves it,
 * same layout, b and key width) back to sorted order, in place.  No counterpart
 * in the reference, whose README describes conversions between sorted order and
 * the layouts but implements only sorted -> layout.  Workspace, stream and ms
 * as for tl_permute (dev_workspace NULL: a cached buffer of
 * tl_unpermute_workspace_bytes, which holds a copy of the array). */
int tl_unpermute_workspace_bytes(int layout, uint64_t n, uint64_t b, uint32_t key_bytes, uint64_t *bytes);
int tl_unpermute(int layout, void *dev_A, uint64_t n, uint64_t b, uint32_t key_bytes, void *dev_workspace,
                 uint64_t workspace_bytes, void *stream, float *ms);

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
/* The same three for the standard vEB layout: buildTable of
 * cpu/src/query-veb.cpp:25-41, and the table set of the reference's CPU query
 * driver cpu/test/query-veb-fixedN.cpp:37-150 (one table per division, here
 * concatenated with table_idx offsets).  tl_query_veb_* and
 * tl_query_veb_nonperfect_* answer queries over a standard vEB layout given
 * these tables (the descent of cpu/src/query-veb.h:41-64 is the same). */
void tl_build_table_std(tl_veb_table *table, uint64_t n, uint32_t d, uint32_t root_depth);
int tl_veb_tables_size_std(uint64_t n, uint32_t *num_tables, uint32_t *table_size, uint32_t *d);
int tl_build_veb_tables_std(uint64_t n, tl_veb_table *tables, uint64_t *idx, uint32_t *table_idx);

/* ---------------------------------------------------------------- queries */
/* Binary search over the sorted array (the comparator the layouts are measured
 * against): dev_answers[i] = index of dev_queries[i] in dev_sorted, or n.
 * Replaces searchAll / binarySearch (gpu/src/binary-search.cuh:27-57) behind
 * timeQuery (:61-118); the reference answers a miss with its predecessor's
 * index (and never ends for a query below A[0]; its driver issues only hits). */
int tl_query_sorted_u32(const uint32_t *dev_sorted, uint64_t n, const uint32_t *dev_queries,
                        uint64_t q, uint64_t *dev_answers, void *stream, float *ms);
int tl_query_sorted_u64(const uint64_t *dev_sorted, uint64_t n, const uint64_t *dev_queries,
                        uint64_t q, uint64_t *dev_answers, void *stream, float *ms);
/* BST and vEB queries: a batch of 2^21 queries or more over a layout of at
 * least 64 MB (BST) or 4 MB (vEB) is first grouped by value, in
 * stream-ordered temporary device memory of about q * (2 w + 8) bytes plus
 * up to 16 MB (w the key width), so that queries close in value share the
 * deep nodes they fetch; the answers keep the batch's order.  If that memory cannot be had, the batch
 * is searched as given.
 *
 * dev_answers[i] = position of dev_queries[i] in the layout, or n.
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

/* ---------------------------------------------------------------- batched mode
 * No counterpart in the reference.  num independent sorted arrays of uneven
 * sizes, concatenated in one device buffer and described by an int64 offset
 * table (offsets[num] = total keys), each permuted to a level-order B-tree of b
 * keys per node (tl_permute's layout, per instance) by one persistent kernel,
 * and queried by a batch of (key, instance) pairs. */
typedef struct tl_batch_plan tl_batch_plan;
/* Builds the per-instance schedules on the device from dev_offsets (num + 1
 * entries) and sizes the workspace (synchronises the stream once). */
int tl_batch_plan_create(const int64_t *dev_offsets, uint32_t num, uint64_t b, uint32_t key_bytes,
                         void *stream, tl_batch_plan **plan);
int tl_batch_plan_destroy(tl_batch_plan *plan);
int tl_batch_workspace_bytes(const tl_batch_plan *plan, uint64_t *bytes);
/* Permutes every instance in place: one memset and one persistent kernel on
 * `stream`, no host synchronisation, capturable in a CUDA graph.  The status of
 * its bounded waits is read by tl_batch_status. */
int tl_batch_permute(const tl_batch_plan *plan, void *dev_keys, void *dev_workspace, uint64_t workspace_bytes,
                     void *stream);
int tl_batch_status(const tl_batch_plan *plan, const void *dev_workspace, void *stream);
int tl_batch_query_workspace_bytes(const tl_batch_plan *plan, uint64_t q, uint64_t *bytes);
/* dev_answers[i] = position of dev_queries[i] inside instance dev_inst[i]'s
 * layout (0-based within the instance), or that instance's n when absent; 0 for
 * an instance id >= num. */
int tl_batch_query(const tl_batch_plan *plan, const void *dev_keys, const void *dev_queries,
                   const uint32_t *dev_inst, uint64_t q, uint64_t *dev_answers, void *dev_workspace,
                   uint64_t workspace_bytes, void *stream, float *ms);
/* Tuning per size class c = floor(log2 n_j), 48 entries each: keys per stream
 * tile (a power of two, 256 .. 96 KB / key_bytes), top levels pinned in shared
 * memory by the query; plus the query work
 * item and the permute block size (256 or 512); 0 / NULL keeps a value.
 * Changing tile sizes rebuilds the plan from dev_offsets. */
int tl_batch_set_tuning(tl_batch_plan *plan, const uint32_t *tile_keys, const uint32_t *pin_levels,
                        uint32_t query_chunk, uint32_t threads, const int64_t *dev_offsets, void *stream);
int tl_batch_get_tuning(const tl_batch_plan *plan, uint32_t *tile_keys, uint32_t *pin_levels,
                        uint32_t *query_chunk, uint32_t *threads);
/* Measures and keeps the best tuning (coordinate descent over the block size,
 * per-class tile sizes, the query work item and per-class pinned levels) on the
 * caller's data; dev_keys must hold the sorted instances and is left sorted.
 * report (optional) receives a JSON summary. */
int tl_batch_autotune(tl_batch_plan *plan, const int64_t *dev_offsets, void *dev_keys, const void *dev_queries,
                      const uint32_t *dev_inst, uint64_t q, void *stream, char *report, uint64_t report_len);

/* ---------------------------------------------------------------- learned-start B-tree query
 * No counterpart in the reference.  A two-stage rank model over the sorted keys:
 * an FP32 root MLP 1 -> 32 -> 32 -> 1 over the normalised key (linear or log2
 * scale) picks one of num_leaves linear segments; a segment predicts the rank
 * and records its largest rank errors below and above the prediction over the
 * keys it was fitted on.  The learned query starts its descent at the deepest
 * subtree whose rank range covers [rank - eps_lo, rank + eps_hi] and falls back to
 * the full search whenever that start cannot decide, so answers equal
 * tl_query_btree_u64's. */
#define TL_RMI_HIDDEN 32
typedef struct tl_rank_model {
    float w1[TL_RMI_HIDDEN], b1[TL_RMI_HIDDEN];                    /* 1 -> 32, ReLU */
    float w2[TL_RMI_HIDDEN][TL_RMI_HIDDEN], b2[TL_RMI_HIDDEN];     /* 32 -> 32, ReLU; w2[out][in] */
    float w3[TL_RMI_HIDDEN], b3;                                   /* 32 -> 1: rank / n */
    float train_loss;                                              /* last training batch's MSE */
    double x_lo, x_scale;          /* x = clamp((f(key) - x_lo) * x_scale, 0, 1) */
    uint64_t n;                    /* number of keys the model was fitted on */
    uint32_t log_feature;          /* f(key) = log2(key + 1) if set, else key */
    uint32_t num_leaves;           /* power of two */
    uint32_t train_root;           /* 0: root network replaced by the identity (ablation) */
    uint32_t reserved;
} tl_rank_model;

typedef struct tl_rank_leaf {
    uint64_t kmin;     /* smallest key of the segment */
    uint64_t base;     /* its rank */
    float slope;       /* ranks per key unit */
    uint32_t eps_lo;   /* largest (prediction - rank) over the segment's keys */
    uint32_t eps_hi;   /* largest (rank - prediction) over the segment's keys */
    uint32_t empty;    /* 1: no key maps to this segment; base and eps_hi
                          then span the ranks between the nearest segments
                          below and above that hold keys (slope 0) */
} tl_rank_leaf;

typedef struct tl_rank_train_config {
    uint32_t num_leaves;   /* e.g. 65536 */
    uint32_t steps;        /* Adam steps on the root network */
    uint32_t batch;        /* (key, rank) samples per step */
    uint32_t log_feature;
    uint32_t train_root;   /* 0 = leaf-only ablation */
    uint32_t monotone;     /* 1: keep w1, w2, w3 >= 0 (the root is then non-decreasing in the key) */
    float lr;              /* Adam step size */
    uint64_t seed;
} tl_rank_train_config;

/* Trains the root network on (key, rank) pairs of the sorted keys (hand-written
 * forward/backward/Adam kernels), fits num_leaves segments and their eps.
 * dev_leaves holds num_leaves entries. */
int tl_rank_model_train(const uint64_t *dev_sorted_keys, uint64_t n, const tl_rank_train_config *cfg,
                        tl_rank_model *model, tl_rank_leaf *dev_leaves, void *stream);
/* Test hook (host only): the root network's output at x[0 .. count) as the
 * inference kernels compute it, from the network compiled into its exact
 * piecewise-linear form; *pieces = the number of linear pieces. */
int tl_debug_rank_model_root(const tl_rank_model *model, const float *x, uint32_t count, float *out,
                             uint32_t *pieces);
/* Inference: dev_rank[i] = predicted rank of dev_keys[i]; dev_eps[i] (optional) =
 * max(eps_lo, eps_hi) of its segment (UINT32_MAX for an empty segment). */
int tl_rank_model_predict(const tl_rank_model *model, const tl_rank_leaf *dev_leaves,
                          const uint64_t *dev_keys, uint64_t q, uint64_t *dev_rank, uint32_t *dev_eps,
                          void *stream);
/* Gradient of the mean squared error of the root network on (x, y) samples
 * (dev_x normalised features, dev_y = rank / n), as computed by the training
 * kernels: host_grad[1153] in the order w1, b1, w2, b2, w3, b3. */
int tl_rank_model_gradient(const tl_rank_model *model, const float *dev_x, const float *dev_y, uint32_t m,
                           float *host_grad, float *host_loss, void *stream);
/* Learned-start query over a B-tree layout of the model's n keys (b*8 a multiple
 * of 16, b <= 32).  dev_stats (optional, 2 words, accumulated): number of
 * queries that fell back to the full search, sum of start depths. */
int tl_query_btree_learned_u64(const uint64_t *dev_layout, uint64_t n, uint64_t b, const tl_rank_model *model,
                               const tl_rank_leaf *dev_leaves, const uint64_t *dev_queries, uint64_t q,
                               uint64_t *dev_answers, unsigned long long *dev_stats, void *stream, float *ms);

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
/* Host replay of tl_permute_algorithm's step list for TL_ALGO_CYCLES or
 * TL_ALGO_HYBRID on n 64-bit words (test hook): the cycle-leader steps, and
 * for the hybrid the perfect front part's involutions as a host permutation;
 * *steps = the number of gather and rotation steps. */
int tl_debug_emulate_algorithm(int layout, int algorithm, uint64_t n, uint64_t b, uint64_t *host_A,
                               uint64_t *steps);
/* Host replay of tl_unpermute's gather on n 64-bit words (test hook). */
int tl_debug_emulate_unpermute(int layout, uint64_t n, uint64_t b, uint64_t *host_A);
/* sizeof of the ABI structs, for bindings to check their mirrors:
 * 0 tl_veb_table, 1 tl_rank_model, 2 tl_rank_leaf, 3 tl_rank_train_config. */
int tl_debug_struct_size(int which);
/* Fixed-direction schedule of the B-tree permutation for (n, b): 0
 * right-to-left, 1 left-to-right (tl_permute_static_ws takes whichever of the
 * two this returns; tl_permute may take the ordered schedule instead). */
int tl_debug_btree_plan(uint64_t n, uint64_t b);
/* Schedule tl_permute takes for (layout, n, b, key_bytes) with a workspace of
 * tl_permute_workspace_bytes: 0 right-to-left, 1 left-to-right, 2 ordered
 * tiles (B-tree from 64 tiles up, BST from 16384), 3 the vEB engine; < 0 on error. */
int tl_debug_permute_plan(int layout, uint64_t n, uint64_t b, uint32_t key_bytes);
/* Kernels the last permutation launched (stream pass and second pass). */
int tl_debug_permute_launches(void);
/* Resident blocks per SM of the stream kernel of `layout` at key_bytes (occupancy check). */
int tl_debug_stream_blocks_per_sm(int layout, uint32_t key_bytes);
/* mode 1: B-tree and BST permutations keep to the fixed-direction schedules
 * (0 and 1 of tl_debug_permute_plan), batched plans built from then on too;
 * mode 2: batched plans built from then on put every instance the ordered
 * schedule applies to on it, whatever it saves; 0 restores the default. */
int tl_debug_set_schedule(int mode);
/* Measurement hook, query kernels: 0 the default; 2 B-tree nodes in 16-byte
 * loads by a thread per query; 3 / 4 vEB two / four descents per thread in
 * lock-step; 5 B-tree a thread per query with 32-byte loads and the top levels
 * pinned in shared memory; 6 B-tree a thread per query with 32-byte loads (in
 * place of a group of lanes per node, for the learned query too); 7 B-tree one
 * 32-byte load per lane of the group (b * w / 32 lanes); 19 BST and vEB
 * batches searched as given, 20 always grouped by value (by default only
 * batches of 2^21 queries or more over BST layouts of 64 MB or more and vEB
 * layouts of 4 MB or more). */
void tl_debug_set_query_variant(int v);
/* Instances of a batched plan on the ordered-tile schedule and their keys: by
 * default those of 64 tiles or more (at the plan's tile size for their size
 * class) whose scratch keys it cuts to 30 % or less. */
int tl_debug_batch_ordered(const tl_batch_plan *plan, uint64_t *instances, uint64_t *keys);
/* Of the last permutation's bounded waits: how many found their flag unset at
 * the first look, and how many polls those took in total. */
int tl_debug_wait_stats(uint64_t *stalled_waits, uint64_t *polls);
/* Keys the permutation of (layout, n, b, key_bytes) moves through its scratch
 * buffer (the second pass reads and writes each once). */
int tl_debug_permute_scratch_keys(int layout, uint64_t n, uint64_t b, uint32_t key_bytes, uint64_t *keys);
/* The ordered-tile tables of (layout, n, b, key_bytes) computed on the host and
 * with their per-tile passes as kernels on `stream` (what a permutation does
 * for a geometry not seen before), uncached, compared entry by entry: 1 equal,
 * 0 different, a negative status when the geometry has no such tables or the
 * kernels could not run. */
int tl_debug_order_tables_match(int layout, uint64_t n, uint64_t b, uint32_t key_bytes, void *stream);
/* tl_permute with library-allocated workspace, reporting the device time of its
 * two passes: phase_ms[0] = setup + stream kernel, phase_ms[1] = the second pass
 * (B-tree: scratch copy kernel, or the fix kernel of the ordered schedule;
 * mvEB: scratch scatter kernel). */
int tl_debug_permute_phases(int layout, void *dev_A, uint64_t n, uint64_t b, uint32_t key_bytes,
                            void *stream, float *phase_ms);

#ifdef __cplusplus
}
#endif
#endif
