// extern "C" surface of libtreelayouts.so (declared in include/tree_layouts.h),
// plus the host-only pieces: mvEB position tables and status plumbing.
#include <atomic>
#include <cstdlib>
#include <cstring>

#include "geometry.cuh"
#include <utility>

#include "internal.h"
#include "learned.h"
#include "stream.cuh"
#include "unpermute.h"
#include "batched.h"

namespace tl {

static thread_local int t_last_cuda_error = 0;
void record_cuda_error(cudaError_t e) { t_last_cuda_error = (int)e; }

static std::atomic<unsigned int> g_spin_limit{1u << 22};  // ~1 s of 256 ns sleeps
static std::atomic<int> g_force_timeout{0};
unsigned int debug_spin_limit() { return g_spin_limit.load(); }
bool debug_force_timeout() { return g_force_timeout.load() != 0; }
void debug_set_wait(unsigned int spin_limit, int force_timeout) {
    g_spin_limit.store(spin_limit ? spin_limit : (1u << 22));
    g_force_timeout.store(force_timeout);
}

int read_error_word(const unsigned int *dev_word, unsigned int *out, cudaStream_t st) {
    // Pageable destination: cudaMemcpyAsync returns once the copy has completed.
    TL_CUDA_TRY(cudaMemcpyAsync(out, dev_word, sizeof(unsigned int), cudaMemcpyDeviceToHost, st));
    TL_CUDA_TRY(cudaStreamSynchronize(st));
    return TL_SUCCESS;
}

// Wait statistics of the last permutation (test and profiling hook).
static std::atomic<unsigned long long> g_stalled_waits{0}, g_stall_polls{0};

void record_wait_stats(const Ctrl *ctrl, cudaStream_t st) {
    unsigned long long v[2] = {0, 0};
    if (cudaMemcpyAsync(v, &ctrl->stalled_waits, sizeof v, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return;
    g_stalled_waits = v[0];
    g_stall_polls = v[1];
}

int sync_and_check(cudaStream_t st) {
    TL_CUDA_TRY(cudaStreamSynchronize(st));
    TL_CUDA_TRY(cudaGetLastError());
    return TL_SUCCESS;
}

// buildTable: gpu/src/query-mveb.cu:25-47 with the mvEB split of
// gpu/src/mveb-cycles.cuh:240-247 (modified), cpu/src/query-veb.cpp:25-41 with
// the standard split (the recursion is the same).
static void build_table(tl_veb_table *table, uint64_t n, uint32_t d, uint32_t root_depth, bool modified) {
    if (n == 1 || d < 2) return;
    uint32_t rd, ld;
    veb_split(d, modified, rd, ld);
    uint64_t root_n = low_mask(rd), leaf_n = low_mask(ld);
    uint32_t i = d - ld;
    table[i].L = leaf_n;
    table[i].R = root_n;
    table[i].D = root_depth;
    build_table(table, root_n, rd, root_depth, modified);
    build_table(&table[i], leaf_n, ld, i + root_depth, modified);
}

// Table-set sizing: gpu/test/query-mveb-fixedN.cu:45-97 (modified),
// cpu/test/query-veb-fixedN.cpp:37-84 (standard).
static void tables_size(uint64_t n, uint32_t &nt, uint32_t &ts, uint32_t &d, bool modified) {
    d = bit_length(n);
    nt = 1;
    ts = d;
    if (n == low_mask(d)) return;
    uint64_t tn = n;
    uint32_t td = d;
    while (td >= 2) {
        uint32_t rd, ld;
        veb_split(td, modified, rd, ld);
        uint64_t r = low_mask(rd), l = low_mask(ld);
        uint64_t nf = (tn - r) / l, inc = tn - r - nf * l;
        if (inc == 0) break;
        uint32_t id = bit_length(inc);
        ++nt;
        ts += id;
        tn = inc;
        td = id;
        if (tn == low_mask(id)) break;
    }
}

}  // namespace tl

using namespace tl;

static inline cudaStream_t S(void *s) { return reinterpret_cast<cudaStream_t>(s); }

extern "C" {

int tl_version(void) { return TL_VERSION; }

const char *tl_status_string(int status) {
    switch (status) {
        case TL_SUCCESS: return "success";
        case TL_ERROR_INVALID_VALUE: return "invalid value";
        case TL_ERROR_CUDA: return "CUDA runtime error";
        case TL_ERROR_TIMEOUT: return "bounded device wait expired";
        case TL_ERROR_OUT_OF_MEMORY: return "out of device memory";
        case TL_ERROR_WORKSPACE_TOO_SMALL: return "workspace too small";
        case TL_ERROR_UNSUPPORTED: return "unsupported size or parameter";
        default: return "unknown status";
    }
}

int tl_last_cuda_error(void) { return t_last_cuda_error; }

// Test hook: bound every device wait to `spin_limit` iterations and, when
// force_timeout is set, make the waits expect a flag value no tile publishes.
int tl_debug_set_wait(unsigned int spin_limit, int force_timeout) {
    debug_set_wait(spin_limit, force_timeout);
    return TL_SUCCESS;
}

int tl_debug_struct_size(int which) {
    switch (which) {
        case 0: return (int)sizeof(tl_veb_table);
        case 1: return (int)sizeof(tl_rank_model);
        case 2: return (int)sizeof(tl_rank_leaf);
        case 3: return (int)sizeof(tl_rank_train_config);
        default: return -1;
    }
}

// Test hook: which fixed-direction B-tree schedule the permutation uses (0:
// right-to-left stream, top tree via scratch; 1: left-to-right stream, last
// level via scratch).
int tl_debug_btree_plan(uint64_t n, uint64_t b) { return btree_plan_of(n, b); }

int tl_debug_permute_plan(int layout, uint64_t n, uint64_t b, uint32_t key_bytes) {
    return permute_plan_of(layout, n, b, key_bytes);
}

int tl_permute_algorithm(int layout, int algorithm, void *dev_A, uint64_t n, uint64_t b, uint32_t key_bytes,
                         void *stream, float *ms) {
    return permute_algorithm(layout, algorithm, dev_A, n, b, key_bytes, S(stream), ms);
}

int tl_unpermute(int layout, void *dev_A, uint64_t n, uint64_t b, uint32_t key_bytes, void *dev_workspace,
                 uint64_t workspace_bytes, void *stream, float *ms) {
    return unpermute(layout, dev_A, n, b, key_bytes, dev_workspace, workspace_bytes, S(stream), ms);
}

int tl_unpermute_workspace_bytes(int layout, uint64_t n, uint64_t b, uint32_t key_bytes, uint64_t *bytes) {
    return unpermute_workspace_bytes(layout, n, b, key_bytes, bytes);
}

int tl_debug_emulate_unpermute(int layout, uint64_t n, uint64_t b, uint64_t *host_A) {
    return emulate_unpermute(layout, n, b, host_A);
}

int tl_debug_stream_blocks_per_sm(int layout, uint32_t key_bytes) { return stream_blocks_per_sm(layout, key_bytes); }

int tl_debug_permute_launches(void) { return last_permute_launches(); }

int tl_debug_set_schedule(int mode) {
    if (mode < 0 || mode > 2) return TL_ERROR_INVALID_VALUE;
    set_schedule_mode(mode);
    return TL_SUCCESS;
}

int tl_debug_wait_stats(uint64_t *stalled_waits, uint64_t *polls) {
    if (!stalled_waits || !polls) return TL_ERROR_INVALID_VALUE;
    *stalled_waits = g_stalled_waits;
    *polls = g_stall_polls;
    return TL_SUCCESS;
}

int tl_debug_batch_ordered(const tl_batch_plan *plan, uint64_t *instances, uint64_t *keys) {
    return batch_ordered(plan, instances, keys);
}

int tl_debug_permute_scratch_keys(int layout, uint64_t n, uint64_t b, uint32_t key_bytes, uint64_t *keys) {
    return permute_scratch_keys(layout, n, b, key_bytes, keys);
}

int tl_debug_order_tables_match(int layout, uint64_t n, uint64_t b, uint32_t key_bytes, void *stream) {
    return debug_order_tables_match(layout, n, b, key_bytes, S(stream));
}

// Measurement hook: query kernel variants (0: the default).
void tl_debug_set_query_variant(int v) { set_query_variant(v); }

// Test hook: host replay of the cycle-leader step list (and, for the hybrid
// BST, the perfect part's two involutions as a host permutation).
int tl_debug_emulate_algorithm(int layout, int algorithm, uint64_t n, uint64_t b, uint64_t *host_A,
                               uint64_t *steps) {
    if (!host_A && n) return TL_ERROR_INVALID_VALUE;
    if (algorithm != TL_ALGO_CYCLES && algorithm != TL_ALGO_HYBRID) return TL_ERROR_INVALID_VALUE;
    if (layout == TL_LAYOUT_BTREE && (b == 0 || b >= (1ull << 20))) return TL_ERROR_INVALID_VALUE;
    if (n <= 1) return TL_SUCCESS;
    uint64_t ni = 0;
    int rc = emulate_cycles(layout, algorithm, n, b, host_A, &ni, steps);
    if (rc || algorithm != TL_ALGO_HYBRID || ni <= 1) return rc;
    // perfect BST of d levels on ranks 1..ni: rank x <-> its d-bit reversal,
    // then x <-> x with its bits below the leading one reversed
    uint32_t d = 0;
    while ((1ull << d) <= ni) ++d;
    auto rev = [](uint64_t x, uint32_t bits) {
        uint64_t r = 0;
        for (uint32_t t = 0; t < bits; ++t) r |= ((x >> t) & 1) << (bits - 1 - t);
        return r;
    };
    for (uint64_t x = 1; x <= ni; ++x) {
        const uint64_t y = rev(x, d);
        if (x < y) std::swap(host_A[x - 1], host_A[y - 1]);
    }
    for (uint64_t x = 1; x <= ni; ++x) {
        uint32_t lb = 0;
        while ((x >> (lb + 1)) != 0) ++lb;  // position of the leading one
        const uint64_t y = ((x >> lb) << lb) | rev(x & ((1ull << lb) - 1), lb);
        if (x < y) std::swap(host_A[x - 1], host_A[y - 1]);
    }
    return TL_SUCCESS;
}

// Test hook: host replay of the permutation's tile schedule (see emulate_permute).
int tl_debug_emulate_permute(int layout, uint64_t n, uint64_t b, uint64_t *host_A, uint64_t *violations) {
    if (n > 0 && !host_A) return TL_ERROR_INVALID_VALUE;
    return emulate_permute(layout, n, b, host_A, violations);
}

int tl_layout_position(int layout, uint64_t n, uint64_t b, uint64_t rank, uint64_t *pos) {
    if (!pos || rank >= n) return TL_ERROR_INVALID_VALUE;
    if (is_veb_layout(layout)) {
        *pos = veb_pos(n, rank, layout == TL_LAYOUT_MVEB);
        return TL_SUCCESS;
    }
    if (layout == TL_LAYOUT_BST) b = 1;
    if (layout != TL_LAYOUT_BTREE && layout != TL_LAYOUT_BST) return TL_ERROR_INVALID_VALUE;
    if (b == 0) return TL_ERROR_INVALID_VALUE;
    BtreeGeom g = make_btree_geom(n, b);
    FastDiv64 fd(b + 1);
    *pos = btree_pos(g, fd, rank);
    return TL_SUCCESS;
}

int tl_permute_workspace_bytes(int layout, uint64_t n, uint64_t b, uint32_t key_bytes, uint64_t *bytes) {
    return permute_workspace_bytes(layout, n, b, key_bytes, bytes);
}

int tl_permute(int layout, void *dev_A, uint64_t n, uint64_t b, uint32_t key_bytes, void *dev_workspace,
               uint64_t workspace_bytes, void *stream, float *ms) {
    return permute(layout, dev_A, n, b, key_bytes, dev_workspace, workspace_bytes, S(stream), ms);
}

// Profiling hook: tl_permute with device times of its two passes
// (phase_ms[0]: control setup + stream kernel, phase_ms[1]: scatter kernel).
int tl_debug_permute_phases(int layout, void *dev_A, uint64_t n, uint64_t b, uint32_t key_bytes, void *stream,
                            float *phase_ms) {
    if (!phase_ms) return TL_ERROR_INVALID_VALUE;
    return permute(layout, dev_A, n, b, key_bytes, nullptr, 0, S(stream), nullptr, phase_ms);
}

int tl_permute_bst_u32(uint32_t *A, uint64_t n, void *s, float *ms) {
    return permute(TL_LAYOUT_BST, A, n, 1, 4, nullptr, 0, S(s), ms);
}
int tl_permute_bst_u64(uint64_t *A, uint64_t n, void *s, float *ms) {
    return permute(TL_LAYOUT_BST, A, n, 1, 8, nullptr, 0, S(s), ms);
}
int tl_permute_btree_u32(uint32_t *A, uint64_t n, uint64_t b, void *s, float *ms) {
    return permute(TL_LAYOUT_BTREE, A, n, b, 4, nullptr, 0, S(s), ms);
}
int tl_permute_btree_u64(uint64_t *A, uint64_t n, uint64_t b, void *s, float *ms) {
    return permute(TL_LAYOUT_BTREE, A, n, b, 8, nullptr, 0, S(s), ms);
}
int tl_permute_mveb_u32(uint32_t *A, uint64_t n, void *s, float *ms) {
    return permute(TL_LAYOUT_MVEB, A, n, 0, 4, nullptr, 0, S(s), ms);
}
int tl_permute_mveb_u64(uint64_t *A, uint64_t n, void *s, float *ms) {
    return permute(TL_LAYOUT_MVEB, A, n, 0, 8, nullptr, 0, S(s), ms);
}

int tl_permute_veb_std_u32(uint32_t *A, uint64_t n, void *s, float *ms) {
    return permute(TL_LAYOUT_VEB, A, n, 0, 4, nullptr, 0, S(s), ms);
}
int tl_permute_veb_std_u64(uint64_t *A, uint64_t n, void *s, float *ms) {
    return permute(TL_LAYOUT_VEB, A, n, 0, 8, nullptr, 0, S(s), ms);
}

void tl_build_table(tl_veb_table *table, uint64_t n, uint32_t d, uint32_t root_depth) {
    if (table) build_table(table, n, d, root_depth, true);
}
void tl_build_table_std(tl_veb_table *table, uint64_t n, uint32_t d, uint32_t root_depth) {
    if (table) build_table(table, n, d, root_depth, false);
}

static int veb_tables_size(uint64_t n, uint32_t *num_tables, uint32_t *table_size, uint32_t *d, bool modified) {
    if (n == 0 || !num_tables || !table_size) return TL_ERROR_INVALID_VALUE;
    uint32_t nt, ts, dd;
    tables_size(n, nt, ts, dd, modified);
    *num_tables = nt;
    *table_size = ts;
    if (d) *d = dd;
    return TL_SUCCESS;
}
int tl_veb_tables_size(uint64_t n, uint32_t *num_tables, uint32_t *table_size, uint32_t *d) {
    return veb_tables_size(n, num_tables, table_size, d, true);
}
int tl_veb_tables_size_std(uint64_t n, uint32_t *num_tables, uint32_t *table_size, uint32_t *d) {
    return veb_tables_size(n, num_tables, table_size, d, false);
}

// Table-set construction: gpu/test/query-mveb-fixedN.cu:130-165 (modified),
// cpu/test/query-veb-fixedN.cpp:116-150 (standard; concatenated with table_idx
// offsets as the GPU driver lays its tables out).
static int build_veb_tables(uint64_t n, tl_veb_table *tables, uint64_t *idx, uint32_t *table_idx, bool modified) {
    if (n == 0 || !tables || !idx || !table_idx) return TL_ERROR_INVALID_VALUE;
    uint32_t nt, ts, d;
    tables_size(n, nt, ts, d, modified);
    memset(tables, 0, ts * sizeof(tl_veb_table));
    build_table(tables, n, d, 0, modified);
    idx[nt - 1] = n;
    table_idx[0] = 0;
    uint64_t tn = n;
    uint32_t td = d;
    for (uint32_t i = 1; i < nt; ++i) {
        table_idx[i] = table_idx[i - 1] + td;
        uint32_t rd, ld;
        veb_split(td, modified, rd, ld);
        uint64_t r = low_mask(rd), l = low_mask(ld);
        uint64_t nf = (tn - r) / l, inc = tn - r - nf * l;
        uint32_t id = bit_length(inc);
        build_table(&tables[table_idx[i]], inc, id, 0, modified);
        idx[i - 1] = n - inc;
        tn = inc;
        td = id;
    }
    return TL_SUCCESS;
}
int tl_build_veb_tables(uint64_t n, tl_veb_table *tables, uint64_t *idx, uint32_t *table_idx) {
    return build_veb_tables(n, tables, idx, table_idx, true);
}
int tl_build_veb_tables_std(uint64_t n, tl_veb_table *tables, uint64_t *idx, uint32_t *table_idx) {
    return build_veb_tables(n, tables, idx, table_idx, false);
}

int tl_batch_plan_create(const int64_t *off, uint32_t num, uint64_t b, uint32_t kb, void *stream,
                         tl_batch_plan **plan) {
    return batch_plan_create(off, num, b, kb, S(stream), plan);
}
int tl_batch_plan_destroy(tl_batch_plan *plan) { return batch_plan_destroy(plan); }
int tl_batch_workspace_bytes(const tl_batch_plan *plan, uint64_t *bytes) { return batch_workspace_bytes(plan, bytes); }
int tl_batch_permute(const tl_batch_plan *plan, void *keys, void *ws, uint64_t wsb, void *stream) {
    return batch_permute(plan, keys, ws, wsb, S(stream));
}
int tl_batch_status(const tl_batch_plan *plan, const void *ws, void *stream) {
    return batch_status(plan, ws, S(stream));
}
int tl_batch_query_workspace_bytes(const tl_batch_plan *plan, uint64_t q, uint64_t *bytes) {
    return batch_query_workspace_bytes(plan, q, bytes);
}
int tl_batch_query(const tl_batch_plan *plan, const void *keys, const void *Q, const uint32_t *inst, uint64_t q,
                   uint64_t *ans, void *ws, uint64_t wsb, void *stream, float *ms) {
    return batch_query(plan, keys, Q, inst, q, ans, ws, wsb, S(stream), ms);
}
int tl_batch_set_tuning(tl_batch_plan *plan, const uint32_t *tile_keys, const uint32_t *pin_levels,
                        uint32_t query_chunk, uint32_t threads, const int64_t *off, void *stream) {
    return batch_set_tuning(plan, tile_keys, pin_levels, query_chunk, threads, off, S(stream));
}
int tl_batch_get_tuning(const tl_batch_plan *plan, uint32_t *tile_keys, uint32_t *pin_levels, uint32_t *query_chunk,
                        uint32_t *threads) {
    return batch_get_tuning(plan, tile_keys, pin_levels, query_chunk, threads);
}
int tl_batch_autotune(tl_batch_plan *plan, const int64_t *off, void *keys, const void *Q, const uint32_t *inst,
                      uint64_t q, void *stream, char *report, uint64_t report_len) {
    return batch_autotune(plan, off, keys, Q, inst, q, S(stream), report, (size_t)report_len);
}

int tl_rank_model_train(const uint64_t *keys, uint64_t n, const tl_rank_train_config *cfg, tl_rank_model *model,
                        tl_rank_leaf *leaves, void *stream) {
    return rank_model_train(keys, n, cfg, model, leaves, S(stream));
}
int tl_debug_rank_model_root(const tl_rank_model *model, const float *x, uint32_t count, float *out,
                             uint32_t *pieces) {
    return rank_model_root_eval(model, x, count, out, pieces);
}

int tl_rank_model_predict(const tl_rank_model *model, const tl_rank_leaf *leaves, const uint64_t *keys, uint64_t q,
                          uint64_t *rank, uint32_t *eps, void *stream) {
    return rank_model_predict(model, leaves, keys, q, rank, eps, S(stream));
}
int tl_rank_model_gradient(const tl_rank_model *model, const float *dx, const float *dy, uint32_t m, float *grad,
                           float *loss, void *stream) {
    return rank_model_gradient(model, dx, dy, m, grad, loss, S(stream));
}
int tl_query_btree_learned_u64(const uint64_t *A, uint64_t n, uint64_t b, const tl_rank_model *model,
                               const tl_rank_leaf *leaves, const uint64_t *Q, uint64_t q, uint64_t *ans,
                               unsigned long long *stats, void *stream, float *ms) {
    return query_btree_learned(A, n, b, model, leaves, Q, q, ans, stats, S(stream), ms);
}

#define TL_Q(NAME, K, KB, LAYOUT, ...)                                                                  \
    int NAME {                                                                                          \
        QueryArgs a{};                                                                                  \
        a.layout = LAYOUT;                                                                              \
        a.key_bytes = KB;                                                                               \
        __VA_ARGS__;                                                                                    \
        return query(a, S(stream), ms);                                                                 \
    }

TL_Q(tl_query_sorted_u32(const uint32_t *L, uint64_t n, const uint32_t *Q, uint64_t q, uint64_t *ans,
                         void *stream, float *ms),
     uint32_t, 4, Q_SORTED, a.layout_keys = L; a.n = n; a.queries = Q; a.q = q; a.answers = ans)
TL_Q(tl_query_sorted_u64(const uint64_t *L, uint64_t n, const uint64_t *Q, uint64_t q, uint64_t *ans,
                         void *stream, float *ms),
     uint64_t, 8, Q_SORTED, a.layout_keys = L; a.n = n; a.queries = Q; a.q = q; a.answers = ans)
TL_Q(tl_query_bst_u32(const uint32_t *L, uint64_t n, const uint32_t *Q, uint64_t q, uint64_t *ans, void *stream,
                      float *ms),
     uint32_t, 4, Q_BST, a.layout_keys = L; a.n = n; a.queries = Q; a.q = q; a.answers = ans)
TL_Q(tl_query_bst_u64(const uint64_t *L, uint64_t n, const uint64_t *Q, uint64_t q, uint64_t *ans, void *stream,
                      float *ms),
     uint64_t, 8, Q_BST, a.layout_keys = L; a.n = n; a.queries = Q; a.q = q; a.answers = ans)
TL_Q(tl_query_btree_u32(const uint32_t *L, uint64_t n, uint64_t b, const uint32_t *Q, uint64_t q, uint64_t *ans,
                        void *stream, float *ms),
     uint32_t, 4, Q_BTREE, a.layout_keys = L; a.n = n; a.b = b; a.queries = Q; a.q = q; a.answers = ans)
TL_Q(tl_query_btree_u64(const uint64_t *L, uint64_t n, uint64_t b, const uint64_t *Q, uint64_t q, uint64_t *ans,
                        void *stream, float *ms),
     uint64_t, 8, Q_BTREE, a.layout_keys = L; a.n = n; a.b = b; a.queries = Q; a.q = q; a.answers = ans)
TL_Q(tl_query_veb_u32(const uint32_t *L, const tl_veb_table *T, uint64_t n, uint32_t d, const uint32_t *Q,
                      uint64_t q, uint64_t *ans, void *stream, float *ms),
     uint32_t, 4, Q_VEB, a.layout_keys = L; a.tables = T; a.n = n; a.d = d; a.queries = Q; a.q = q;
     a.answers = ans)
TL_Q(tl_query_veb_u64(const uint64_t *L, const tl_veb_table *T, uint64_t n, uint32_t d, const uint64_t *Q,
                      uint64_t q, uint64_t *ans, void *stream, float *ms),
     uint64_t, 8, Q_VEB, a.layout_keys = L; a.tables = T; a.n = n; a.d = d; a.queries = Q; a.q = q;
     a.answers = ans)
TL_Q(tl_query_veb_nonperfect_u32(const uint32_t *L, const tl_veb_table *T, const uint64_t *idx,
                                 const uint32_t *tidx, uint64_t n, uint32_t d, uint32_t nt, const uint32_t *Q,
                                 uint64_t q, uint64_t *ans, void *stream, float *ms),
     uint32_t, 4, Q_VEB_NP, a.layout_keys = L; a.tables = T; a.idx = idx; a.table_idx = tidx; a.n = n; a.d = d;
     a.num_tables = nt; a.queries = Q; a.q = q; a.answers = ans)
TL_Q(tl_query_veb_nonperfect_u64(const uint64_t *L, const tl_veb_table *T, const uint64_t *idx,
                                 const uint32_t *tidx, uint64_t n, uint32_t d, uint32_t nt, const uint64_t *Q,
                                 uint64_t q, uint64_t *ans, void *stream, float *ms),
     uint64_t, 8, Q_VEB_NP, a.layout_keys = L; a.tables = T; a.idx = idx; a.table_idx = tidx; a.n = n; a.d = d;
     a.num_tables = nt; a.queries = Q; a.q = q; a.answers = ans)

}  // extern "C"
