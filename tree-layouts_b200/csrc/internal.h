// Host-side helpers shared by the library's translation units.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/tree_layouts.h"

namespace tl {

void record_cuda_error(cudaError_t e);

// The two van Emde Boas layouts share one permutation engine (split rule aside).
inline bool is_veb_layout(int layout) { return layout == TL_LAYOUT_MVEB || layout == TL_LAYOUT_VEB; }

#define TL_CUDA_TRY(expr)                       \
    do {                                        \
        cudaError_t tl_e_ = (expr);             \
        if (tl_e_ != cudaSuccess) {             \
            ::tl::record_cuda_error(tl_e_);     \
            return TL_ERROR_CUDA;               \
        }                                       \
    } while (0)

// Bounded-wait knobs (fault-injection tests shrink the bound and make waits miss).
unsigned int debug_spin_limit();
bool debug_force_timeout();
void debug_set_wait(unsigned int spin_limit, int force_timeout);

// Optional device-time measurement on a stream with CUDA events.
class EventTimer {
   public:
    EventTimer(bool on, cudaStream_t st) : on_(on), st_(st) {
        if (on_) {
            cudaEventCreate(&a_);
            cudaEventCreate(&b_);
        }
    }
    ~EventTimer() {
        if (on_) {
            cudaEventDestroy(a_);
            cudaEventDestroy(b_);
            if (m_) cudaEventDestroy(m_);
        }
    }
    void start() {
        if (on_) cudaEventRecord(a_, st_);
    }
    void stop() {
        if (on_) cudaEventRecord(b_, st_);
    }
    // Optional split point: elapsed_split() returns [start, mid] and [mid, stop].
    void mid() {
        if (on_) {
            if (!m_) cudaEventCreate(&m_);
            cudaEventRecord(m_, st_);
        }
    }
    void elapsed_split(float *first, float *second) {
        *first = *second = 0.f;
        if (on_ && m_) {
            cudaEventSynchronize(b_);
            cudaEventElapsedTime(first, a_, m_);
            cudaEventElapsedTime(second, m_, b_);
        }
    }
    float elapsed() {
        float ms = 0.f;
        if (on_) {
            cudaEventSynchronize(b_);
            cudaEventElapsedTime(&ms, a_, b_);
        }
        return ms;
    }

   private:
    bool on_;
    cudaStream_t st_;
    cudaEvent_t a_{}, b_{}, m_{};
};

// Reads a device word written by the preceding work on `st` (blocks the host).
int read_error_word(const unsigned int *dev_word, unsigned int *out, cudaStream_t st);
// A cached device buffer of at least `bytes` for one synchronous call (nullptr
// when none can be had); give it back with workspace_release once the call's
// work on its stream has finished.
void *workspace_acquire(size_t bytes);
void workspace_release(void *p);
// Raises the current device's default pool release threshold (once per device)
// so that stream-ordered allocations are reused across calls.
void keep_pool_memory();
int sync_and_check(cudaStream_t st);
struct Ctrl;
// Keeps the wait statistics of a permutation's control block (tl_debug_wait_stats).
void record_wait_stats(const Ctrl *ctrl, cudaStream_t st);

int permute_workspace_bytes(int layout, uint64_t n, uint64_t b, uint32_t key_bytes, uint64_t *bytes);
// The workspace of the fixed-direction schedules (what permute needs when told
// not to take the ordered one).
int permute_workspace_bytes_fixed(int layout, uint64_t n, uint64_t b, uint32_t key_bytes, uint64_t *bytes);
int btree_plan_of(uint64_t n, uint64_t b);
int permute_plan_of(int layout, uint64_t n, uint64_t b, uint32_t key_bytes);
int permute_algorithm(int layout, int algorithm, void *dev_A, uint64_t n, uint64_t b, uint32_t key_bytes,
                      cudaStream_t st, float *ms);
// Debug schedule mode (tl_debug_set_schedule): 0 default, 1 fixed directions
// only, 2 batched plans order every instance the ordered schedule applies to.
void set_schedule_mode(int mode);
bool fixed_schedule_only();
bool ordered_schedule_forced();
int stream_blocks_per_sm(int layout, uint32_t key_bytes);
int last_permute_launches();
int permute_scratch_keys(int layout, uint64_t n, uint64_t b, uint32_t key_bytes, uint64_t *keys);
int debug_order_tables_match(int layout, uint64_t n, uint64_t b, uint32_t key_bytes, cudaStream_t st);
int emulate_permute(int layout, uint64_t n, uint64_t b, uint64_t *A, uint64_t *violations);
// query.cu: kernel selection for measurements (0: the default)
void set_query_variant(int v);
int query_variant();
// cycles.cu: the cycle-leader family (and the hybrid BST's last level); for
// the hybrid *perfect = keys of the front part the involutions finish
int permute_cycles(int layout, int algorithm, void *dev_A, uint64_t n, uint64_t b, uint32_t key_bytes,
                   cudaStream_t st, uint64_t *perfect);
int emulate_cycles(int layout, int algorithm, uint64_t n, uint64_t b, uint64_t *A, uint64_t *perfect,
                   uint64_t *steps);
int permute(int layout, void *dev_A, uint64_t n, uint64_t b, uint32_t key_bytes, void *dev_ws,
            uint64_t ws_bytes, cudaStream_t st, float *ms, float *phase_ms = nullptr, bool allow_ordered = true);

enum QueryLayout { Q_BST = 0, Q_BTREE = 1, Q_VEB = 2, Q_VEB_NP = 3, Q_SORTED = 4 };
struct QueryArgs {
    int layout;
    uint32_t key_bytes;
    const void *layout_keys;
    uint64_t n, b;
    const tl_veb_table *tables;
    const uint64_t *idx;
    const uint32_t *table_idx;
    uint32_t d, num_tables;
    const void *queries;
    uint64_t q;
    uint64_t *answers;
};
int query(const QueryArgs &a, cudaStream_t st, float *ms);

}  // namespace tl
