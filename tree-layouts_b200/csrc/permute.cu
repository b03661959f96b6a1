// In-place permutations sorted -> {B-tree, BST, mvEB} for sm_100a.
//
// Every layout is a pure index permutation with the same two-part structure:
// most keys belong to "bulk" runs (the leaf level of a B-tree, the bottom-level
// subtrees of an mvEB) that land at a position >= their source position, and a
// minority (the separators above them) land further left.  The permutation is
// therefore done in two kernels instead of the reference's chain of cycle-leader
// and reversal launches:
//
//  1. stream: one pass over the array from the right end to the left, one tile
//     per ticket.  A tile is read into shared memory, flagged as read, and its
//     bulk keys are stored straight to their final positions once the tiles
//     under those positions have been read.  Separators go to a scratch buffer.
//  2. scatter: the scratch buffer is written to its final positions (out of
//     place, every destination is free by then).
//
// DRAM traffic is 2*n*w for the stream plus 2*w per separator: n/(b+1)
// separators for a perfect B-tree, about n/2^8 for an mvEB.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <vector>

#include "btree_plan.cuh"
#include "geometry.cuh"
#include "internal.h"
#include "stream.cuh"

namespace tl {

constexpr int kStreamThreads = 256;
constexpr uint32_t kUnitMaxLevels = 8;

template <typename K>
constexpr uint64_t stream_tile_keys() {
    return 32768 / sizeof(K);
}

static inline uint64_t align_up(uint64_t x, uint64_t a) { return (x + a - 1) / a * a; }

template <typename K>
__global__ void __launch_bounds__(kStreamThreads)
btree_stream_kernel(K *__restrict__ A, K *__restrict__ scr, BtreeStream S, Ctrl *ctrl, WaitCfg wc,
                    unsigned int *flags) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    K *sm = reinterpret_cast<K *>(smem_raw);
    __shared__ unsigned long long s_ticket;
    __shared__ int s_ok;
    for (;;) {
        unsigned long long t = next_ticket(ctrl, &s_ticket);
        if (t >= S.ntiles) break;
        btree_stream_tile(S, A, scr, flags, ctrl, wc, btree_tile_of_ticket(S, t), sm, &s_ok);
    }
}

// kQueue: the per-warp deferred queues exist (b > 1, or plan L); binary trees
// under plan R use the branch-free path and no shared memory, which leaves more
// blocks resident.
template <typename K, bool kQueue>
__global__ void __launch_bounds__(kScatterThreads, kQueue ? 6 : 8)
btree_scatter_kernel(K *__restrict__ A, const K *__restrict__ scr, BtreeStream S) {
    __shared__ K qval[kQueue ? (kScatterThreads / 32) * kDeferCap : 1];
    __shared__ uint16_t qoff[kQueue ? (kScatterThreads / 32) * kDeferCap : 1];
    for (uint64_t c0 = (uint64_t)blockIdx.x * kScatterChunk; c0 < S.nscratch;
         c0 += (uint64_t)gridDim.x * kScatterChunk)
        btree_scatter_chunk<K, !kQueue>(S, A, scr, c0, qval, qoff);
}

// ---------------------------------------------------------------- mvEB stream
struct MvebParams {
    MvebPlan plan;
    // inv_perm_U[q]: sorted rank (within a unit of U levels) at unit position q.
    unsigned char inv1[1], inv2[3], inv4[15], inv8[255];
};

TL_HD int mveb_region_of_tile(const MvebPlan &P, uint64_t k) {
    int r = 0;
    while (r + 1 < P.nreg && k >= P.reg[r + 1].tile_base) ++r;
    return r;
}

TL_HD uint64_t mveb_tile_of(const MvebPlan &P, uint64_t x) {
    int r = 0;
    while (r + 1 < P.nreg && x >= P.reg[r + 1].src) ++r;
    const MvebRegion &R = P.reg[r];
    return R.tile_base + (x - R.src) / R.tile_len;
}

TL_HD void mveb_tile(const MvebPlan &P, uint64_t k, int &ri, uint64_t &p0, uint64_t &p1) {
    ri = mveb_region_of_tile(P, k);
    const MvebRegion &R = P.reg[ri];
    p0 = R.src + (k - R.tile_base) * R.tile_len;
    p1 = R.src + R.len < p0 + R.tile_len ? R.src + R.len : p0 + R.tile_len;
}

// Groups [g0, g1) of a unit-region tile; the last group of a perfect segment has
// no separator.
TL_HD void mveb_tile_groups(const MvebRegion &R, uint64_t p0, uint64_t p1, uint64_t &g0, uint64_t &g1) {
    const uint64_t u = (1ull << R.U) - 1;
    g0 = (p0 - R.src) >> R.U;
    g1 = (p1 - R.src + u) >> R.U;
}

TL_HD bool mveb_tile_wait(const MvebPlan &P, const MvebRegion &R, uint64_t p0, uint64_t p1, uint64_t &k_lo,
                          uint64_t &k_hi) {
    if (R.U == 0) return false;
    uint64_t g0, g1;
    mveb_tile_groups(R, p0, p1, g0, g1);
    const uint64_t d0 = mveb_unit_dst(R, g0);
    const uint64_t d1 = mveb_unit_dst(R, g1 - 1) + (1ull << R.U) - 1;
    const uint64_t lo = d0 > p1 ? d0 : p1;
    if (lo >= d1) return false;
    k_lo = mveb_tile_of(P, lo);
    k_hi = mveb_tile_of(P, d1 - 1);
    return true;
}

// Sorted rank held by scratch slot s, or ~0 for an unused slot.
TL_HD uint64_t mveb_slot_rank(const MvebPlan &P, uint64_t s) {
    int r = 0;
    while (r + 1 < P.nreg && s >= P.reg[r + 1].slot_base) ++r;
    const MvebRegion &R = P.reg[r];
    const uint64_t rank =
        R.U ? R.src + ((s - R.slot_base) << R.U) + ((1ull << R.U) - 1) : R.src + (s - R.slot_base);
    return rank < R.src + R.len ? rank : ~0ull;
}

template <typename K>
__global__ void __launch_bounds__(kStreamThreads)
mveb_stream_kernel(K *__restrict__ A, K *__restrict__ scr, const __grid_constant__ MvebParams prm,
                   Ctrl *ctrl, WaitCfg wc, unsigned int *flags) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    K *sm = reinterpret_cast<K *>(smem_raw);
    __shared__ unsigned long long s_ticket;
    __shared__ int s_ok;
    __shared__ unsigned char s_inv[256];
    const MvebPlan &P = prm.plan;
    const uint64_t ntiles = P.total_tiles;
    int loaded_U = -1;
    for (;;) {
        unsigned long long t = next_ticket(ctrl, &s_ticket);
        if (t >= ntiles) break;
        const uint64_t k = ntiles - 1 - t;
        int ri;
        uint64_t p0, p1;
        mveb_tile(P, k, ri, p0, p1);
        const MvebRegion &R = P.reg[ri];
        if ((int)R.U != loaded_U && R.U) {  // block-uniform: unit tables for this height
            const unsigned char *src = R.U == 8 ? prm.inv8 : R.U == 4 ? prm.inv4 : R.U == 2 ? prm.inv2 : prm.inv1;
            for (uint32_t q = threadIdx.x; q < (1u << R.U) - 1; q += blockDim.x) s_inv[q] = src[q];
            loaded_U = R.U;
        }
        const uint64_t base = load_tile(A, p0, p1, sm);
        publish_read(&flags[k], wc);
        if (R.U == 0) {
            for (uint64_t x = p0 + threadIdx.x; x < p1; x += blockDim.x)
                scr[R.slot_base + (x - R.src)] = sm[x - base];
            continue;
        }
        uint64_t k_lo, k_hi;
        if (mveb_tile_wait(P, R, p0, p1, k_lo, k_hi) &&
            !wait_tiles(flags, (long long)k_lo, (long long)k_hi, ctrl, wc, &s_ok))
            continue;
        const uint32_t U = R.U;
        const uint64_t u = (1ull << U) - 1;
        uint64_t g0, g1;
        mveb_tile_groups(R, p0, p1, g0, g1);
        const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
        for (uint64_t gi = g0 + warp; gi < g1; gi += nwarps) {
            const uint64_t gsrc = R.src + (gi << U) - base;
            const uint64_t dst = mveb_unit_dst(R, gi);
            for (uint32_t q = lane; q < u; q += 32) A[dst + q] = sm[gsrc + s_inv[q]];
            if (lane == 0 && R.src + (gi << U) + u < R.src + R.len) scr[R.slot_base + gi] = sm[gsrc + u];
        }
    }
}

template <typename K>
__global__ void __launch_bounds__(kScatterThreads)
mveb_scatter_kernel(K *__restrict__ A, const K *__restrict__ scr, const __grid_constant__ MvebParams prm) {
    const MvebPlan &P = prm.plan;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    uint64_t s = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    for (; s + 3 * stride < P.total_slots; s += 4 * stride) {
        K v[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) v[u] = __ldcs(scr + s + u * stride);
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const uint64_t rank = mveb_slot_rank(P, s + u * stride);
            if (rank != ~0ull) A[mveb_pos(P.n, rank)] = v[u];
        }
    }
    for (; s < P.total_slots; s += stride) {
        const uint64_t rank = mveb_slot_rank(P, s);
        if (rank != ~0ull) A[mveb_pos(P.n, rank)] = scr[s];
    }
}

// ---------------------------------------------------------------- host side
static void fill_unit_tables(MvebParams &prm) {
    auto fill = [](unsigned char *inv, uint32_t U) {
        uint64_t m = (1ull << U) - 1;
        for (uint64_t s = 0; s < m; ++s) inv[mveb_pos(m, s)] = (unsigned char)s;
    };
    fill(prm.inv1, 1);
    fill(prm.inv2, 2);
    fill(prm.inv4, 4);
    fill(prm.inv8, 8);
}

struct PermutePlan {
    int layout = 0;
    uint32_t key_bytes = 8;
    uint64_t n = 0, b = 1;
    uint64_t tile_keys = 0, ntiles = 0, scratch_keys = 0;
    BtreeStream bs;
    MvebParams mp;
    uint64_t off_flags = 0, off_ctrl = 0, bytes = 0;
};

static int make_plan(int layout, uint64_t n, uint64_t b, uint32_t key_bytes, PermutePlan &pl) {
    if (key_bytes != 4 && key_bytes != 8) return TL_ERROR_INVALID_VALUE;
    if (layout == TL_LAYOUT_BST) b = 1;
    if (layout == TL_LAYOUT_BTREE && b == 0) return TL_ERROR_INVALID_VALUE;
    if (layout < TL_LAYOUT_BST || layout > TL_LAYOUT_MVEB) return TL_ERROR_INVALID_VALUE;
    pl.layout = layout;
    pl.key_bytes = key_bytes;
    pl.n = n;
    pl.b = b;
    pl.tile_keys = 32768 / key_bytes;
    if (layout == TL_LAYOUT_MVEB) {
        if (n >= (1ull << 62)) return TL_ERROR_UNSUPPORTED;
        pl.mp.plan = make_mveb_plan(n, kUnitMaxLevels, pl.tile_keys);
        fill_unit_tables(pl.mp);
        pl.ntiles = pl.mp.plan.total_tiles;
        pl.scratch_keys = pl.mp.plan.total_slots;
    } else {
        if (b >= (1ull << 31)) return TL_ERROR_UNSUPPORTED;
        pl.bs.g = make_btree_geom(n, b);
        pl.bs.fd = FastDiv64(b + 1);
        pl.bs.fd32 = FastDiv32((uint32_t)(b + 1));
        pl.bs.tile_keys = pl.tile_keys;
        pl.ntiles = (n + pl.tile_keys - 1) / pl.tile_keys;
        pl.bs.ntiles = pl.ntiles;
        btree_choose_plan(pl.bs);
        pl.scratch_keys = pl.bs.nscratch;
    }
    pl.off_flags = align_up(pl.scratch_keys * key_bytes, 256);
    pl.off_ctrl = pl.off_flags + align_up(pl.ntiles * sizeof(unsigned int), 256);
    pl.bytes = pl.off_ctrl + align_up(sizeof(Ctrl), 256);
    return TL_SUCCESS;
}

static int g_sm_count = 0;
static std::once_flag g_props_once;
static int sm_count() {
    std::call_once(g_props_once, [] {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&g_sm_count, cudaDevAttrMultiProcessorCount, dev);
        if (g_sm_count <= 0) g_sm_count = 148;
    });
    return g_sm_count;
}

template <typename K>
static int launch_permute(const PermutePlan &pl, K *A, char *ws, cudaStream_t st, EventTimer &timer) {
    K *scr = reinterpret_cast<K *>(ws);
    unsigned int *flags = reinterpret_cast<unsigned int *>(ws + pl.off_flags);
    Ctrl *ctrl = reinterpret_cast<Ctrl *>(ws + pl.off_ctrl);
    WaitCfg wc;
    wc.flag_value = 1;
    wc.wait_value = debug_force_timeout() ? 0xFFFFFFFFu : 1u;  // forced: no tile ever publishes it
    wc.spin_limit = debug_spin_limit();
    // flags and control block are contiguous: one stream-ordered memset clears both
    TL_CUDA_TRY(cudaMemsetAsync(flags, 0, pl.bytes - pl.off_flags, st));
    const size_t smem = (size_t)pl.tile_keys * sizeof(K) + 16;
    const int smx = sm_count();
    if (pl.layout == TL_LAYOUT_MVEB) {
        auto kern = mveb_stream_kernel<K>;
        TL_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        int per_sm = 0;
        TL_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kStreamThreads, smem));
        uint64_t grid = std::min<uint64_t>((uint64_t)std::max(per_sm, 1) * smx, std::max<uint64_t>(pl.ntiles, 1));
        if (pl.ntiles) kern<<<(unsigned)grid, kStreamThreads, smem, st>>>(A, scr, pl.mp, ctrl, wc, flags);
        TL_CUDA_TRY(cudaGetLastError());
        timer.mid();
        if (pl.scratch_keys) {
            int sper = 0;
            TL_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&sper, mveb_scatter_kernel<K>,
                                                                      kScatterThreads, 0));
            uint64_t sg = std::min<uint64_t>((pl.scratch_keys + kScatterThreads - 1) / kScatterThreads,
                                             (uint64_t)std::max(sper, 1) * smx);
            mveb_scatter_kernel<K><<<(unsigned)sg, kScatterThreads, 0, st>>>(A, scr, pl.mp);
            TL_CUDA_TRY(cudaGetLastError());
        }
    } else {
        auto kern = btree_stream_kernel<K>;
        TL_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        int per_sm = 0;
        TL_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kStreamThreads, smem));
        uint64_t grid = std::min<uint64_t>((uint64_t)std::max(per_sm, 1) * smx, std::max<uint64_t>(pl.ntiles, 1));
        if (pl.ntiles) kern<<<(unsigned)grid, kStreamThreads, smem, st>>>(A, scr, pl.bs, ctrl, wc, flags);
        TL_CUDA_TRY(cudaGetLastError());
        timer.mid();
        if (pl.scratch_keys) {
            // one wave of resident blocks striding over the chunks: a second,
            // partial wave would leave the tail of the pass under-occupied
            const bool queue = !(pl.bs.g.b == 1 && pl.bs.plan == PLAN_R);
            auto skern = queue ? btree_scatter_kernel<K, true> : btree_scatter_kernel<K, false>;
            int sper = 0;
            TL_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&sper, skern, kScatterThreads, 0));
            uint64_t sg = std::min<uint64_t>((pl.scratch_keys + kScatterChunk - 1) / kScatterChunk,
                                             (uint64_t)std::max(sper, 1) * smx);
            skern<<<(unsigned)sg, kScatterThreads, 0, st>>>(A, scr, pl.bs);
            TL_CUDA_TRY(cudaGetLastError());
        }
    }
    return TL_SUCCESS;
}

// The library's own workspaces come from the device's stream-ordered pool; keep
// freed blocks in the pool (instead of returning them to the driver at every
// synchronisation) so repeated calls reuse them without re-mapping memory.
static void keep_pool_memory() {
    static std::once_flag once[64];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return;
    std::call_once(once[dev], [dev] {
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
            uint64_t keep = UINT64_MAX;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        }
    });
}

int btree_plan_of(uint64_t n, uint64_t b) {
    PermutePlan pl;
    if (make_plan(TL_LAYOUT_BTREE, n, b, 8, pl)) return -1;
    return pl.bs.plan;
}

int permute_workspace_bytes(int layout, uint64_t n, uint64_t b, uint32_t key_bytes, uint64_t *bytes) {
    if (!bytes) return TL_ERROR_INVALID_VALUE;
    PermutePlan pl;
    int rc = make_plan(layout, n, b, key_bytes, pl);
    if (rc) return rc;
    *bytes = pl.bytes;
    return TL_SUCCESS;
}

int permute(int layout, void *dev_A, uint64_t n, uint64_t b, uint32_t key_bytes, void *dev_ws,
            uint64_t ws_bytes, cudaStream_t st, float *ms, float *phase_ms) {
    if (n > 0 && !dev_A) return TL_ERROR_INVALID_VALUE;
    if (reinterpret_cast<uintptr_t>(dev_A) % (key_bytes ? key_bytes : 1)) return TL_ERROR_INVALID_VALUE;
    if (dev_ws && reinterpret_cast<uintptr_t>(dev_ws) % 256) return TL_ERROR_INVALID_VALUE;
    PermutePlan pl;
    int rc = make_plan(layout, n, b, key_bytes, pl);
    if (rc) return rc;
    if (n <= 1) {
        if (ms) *ms = 0.f;
        return TL_SUCCESS;
    }
    if (dev_ws && ws_bytes < pl.bytes) return TL_ERROR_WORKSPACE_TOO_SMALL;
    EventTimer timer(ms != nullptr || phase_ms != nullptr, st);
    char *ws = static_cast<char *>(dev_ws);
    bool owned = false;
    if (!ws) {
        keep_pool_memory();
        if (cudaMallocAsync(reinterpret_cast<void **>(&ws), pl.bytes, st) != cudaSuccess) {
            record_cuda_error(cudaGetLastError());
            return TL_ERROR_OUT_OF_MEMORY;
        }
        owned = true;
    }
    timer.start();
    rc = key_bytes == 8 ? launch_permute<uint64_t>(pl, static_cast<uint64_t *>(dev_A), ws, st, timer)
                        : launch_permute<uint32_t>(pl, static_cast<uint32_t *>(dev_A), ws, st, timer);
    timer.stop();
    unsigned int err = 0;
    if (rc == TL_SUCCESS) {
        Ctrl *ctrl = reinterpret_cast<Ctrl *>(ws + pl.off_ctrl);
        rc = read_error_word(&ctrl->error, &err, st);
    }
    if (owned) cudaFreeAsync(ws, st);
    if (rc == TL_SUCCESS) rc = sync_and_check(st);
    if (rc == TL_SUCCESS && err) rc = TL_ERROR_TIMEOUT;
    if (rc == TL_SUCCESS && ms) *ms = timer.elapsed();
    if (rc == TL_SUCCESS && phase_ms) timer.elapsed_split(&phase_ms[0], &phase_ms[1]);
    return rc;
}

// Host replay of the stream + scatter passes on a host array, one tile at a time
// in ticket order, using the same index helpers as the kernels.  Besides the
// result it counts protocol violations: a tile reading a position that was
// already overwritten, a store outside the tile's own source that is not covered
// by the tiles it waits for, a wait on a tile with a later ticket, and a final
// position or scratch slot written other than exactly once.  Test hook only.
int emulate_permute(int layout, uint64_t n, uint64_t b, uint64_t *A, uint64_t *violations) {
    PermutePlan pl;
    int rc = make_plan(layout, n, b, 8, pl);
    if (rc) return rc;
    uint64_t viol = 0;
    if (n > 1) {
        std::vector<uint64_t> scr(pl.scratch_keys, 0), tile(pl.tile_keys + 1);
        std::vector<uint8_t> readk(pl.ntiles, 0), written(n, 0);
        std::vector<uint32_t> slot_writes(pl.scratch_keys, 0), pos_writes(n, 0);
        const bool mv = pl.layout == TL_LAYOUT_MVEB;
        const MvebPlan &P = pl.mp.plan;
        auto tile_of = [&](uint64_t d) { return mv ? mveb_tile_of(P, d) : d / pl.tile_keys; };
        for (uint64_t t = 0; t < pl.ntiles; ++t) {
            const uint64_t k = mv ? pl.ntiles - 1 - t : btree_tile_of_ticket(pl.bs, t);
            uint64_t p0, p1, k_lo = 0, k_hi = 0;
            int ri = 0;
            if (mv) mveb_tile(P, k, ri, p0, p1); else btree_tile(pl.bs, k, p0, p1);
            for (uint64_t x = p0; x < p1; ++x) {
                if (written[x]) ++viol;
                tile[x - p0] = A[x];
            }
            readk[k] = 1;
            const bool wait = mv ? mveb_tile_wait(P, P.reg[ri], p0, p1, k_lo, k_hi)
                                 : btree_tile_wait(pl.bs, p0, p1, k_lo, k_hi);
            if (wait)
                for (uint64_t kk = k_lo; kk <= k_hi; ++kk) {
                    const bool earlier = (mv || pl.bs.plan == PLAN_R) ? kk > k : kk < k;
                    if (!earlier || !readk[kk]) ++viol;
                }
            auto W = [&](uint64_t d, uint64_t v) {
                if (d >= n) { ++viol; return; }
                const uint64_t kd = tile_of(d);
                if (kd != k && !(wait && kd >= k_lo && kd <= k_hi)) ++viol;
                if (!readk[kd]) ++viol;
                A[d] = v;
                written[d] = 1;
                ++pos_writes[d];
            };
            auto SC = [&](uint64_t s, uint64_t v) {
                if (s >= scr.size()) { ++viol; return; }
                scr[s] = v;
                ++slot_writes[s];
            };
            if (!mv) {
                const TileDiv td = btree_tile_div(pl.bs, p0);
                const Regime RG = btree_stream_regime(pl.bs, p0, p1);
                for (uint64_t x = p0; x < p1; ++x) {
                    uint64_t idx, idx2, idx3;
                    const bool direct = btree_place_tile(pl.bs, td, x, idx);
                    if (direct != btree_place(pl.bs, x, idx2) || idx != idx2) ++viol;  // fast path == reference form
                    if (RG.kind && (btree_regime_place(pl.bs, RG, (uint32_t)(x - p0), idx3) != direct || idx3 != idx))
                        ++viol;
                    if (direct) W(idx, tile[x - p0]); else SC(idx, tile[x - p0]);
                }
            } else {
                const MvebRegion &R = P.reg[ri];
                if (R.U == 0) {
                    for (uint64_t x = p0; x < p1; ++x) SC(R.slot_base + (x - R.src), tile[x - p0]);
                } else {
                    const unsigned char *inv = R.U == 8 ? pl.mp.inv8 : R.U == 4 ? pl.mp.inv4
                                             : R.U == 2 ? pl.mp.inv2 : pl.mp.inv1;
                    const uint64_t u = (1ull << R.U) - 1;
                    uint64_t g0, g1;
                    mveb_tile_groups(R, p0, p1, g0, g1);
                    for (uint64_t gi = g0; gi < g1; ++gi) {
                        const uint64_t gsrc = R.src + (gi << R.U) - p0;
                        const uint64_t dst = mveb_unit_dst(R, gi);
                        for (uint64_t q = 0; q < u; ++q) {
                            if (gsrc + inv[q] >= p1 - p0) { ++viol; continue; }
                            W(dst + q, tile[gsrc + inv[q]]);
                        }
                        if (R.src + (gi << R.U) + u < R.src + R.len) SC(R.slot_base + gi, tile[gsrc + u]);
                    }
                }
            }
        }
        if (!mv) {
            for (uint64_t c = 0; c < pl.bs.nscratch; ++c) {
                if (slot_writes[c] != 1) ++viol;
                const uint64_t cc0 = c - c % kScatterChunk;
                const ScatterDiv sd = btree_scatter_div(pl.bs, cc0);
                const uint64_t d = btree_slot_dest(pl.bs, c);
                if (btree_slot_dest_tile(pl.bs, sd, c) != d) ++viol;  // fast path == reference form
                const Regime RG = btree_scatter_regime(pl.bs, cc0, std::min(pl.bs.nscratch, cc0 + kScatterChunk));
                if (RG.kind == 1 && btree_regime_slot_dest(pl.bs, RG, cc0, (uint32_t)(c - cc0)) != d) ++viol;
                if (d >= n) { ++viol; continue; }
                A[d] = scr[c];
                ++pos_writes[d];
            }
        } else {
            for (uint64_t s2 = 0; s2 < P.total_slots; ++s2) {
                const uint64_t rank = mveb_slot_rank(P, s2);
                if (rank == ~0ull) { if (slot_writes[s2]) ++viol; continue; }
                if (slot_writes[s2] != 1) ++viol;
                const uint64_t d = mveb_pos(n, rank);
                A[d] = scr[s2];
                ++pos_writes[d];
            }
        }
        for (uint64_t d = 0; d < n; ++d)
            if (pos_writes[d] != 1) ++viol;
    }
    if (violations) *violations = viol;
    return TL_SUCCESS;
}

}  // namespace tl
