// Reverse permutations: a B-tree, BST, mvEB or standard-vEB layout back to
// sorted order, in place.  The reference converts only from sorted order to the
// layouts; this is the other direction of the same index maps.
//
// Every sorted tile draws its keys from the layout the way the forward pass
// sends them: its bulk keys from one contiguous range of the layout (a B-tree's
// last level; whole vEB units) and its top keys from one contiguous run per
// level of the top tree (B-tree) or one separator per unit (vEB), so the same
// per-tile helpers describe the gather.  The layout is first copied to the
// workspace (a stream-ordered device copy); then one kernel gathers each sorted
// tile from the copy into shared memory in sorted order and stores it with
// whole-tile coalesced writes.  Traffic: 2*n*w for the copy plus 2*n*w for the
// gather; reads of the gather are contiguous runs.
#include <algorithm>
#include <mutex>
#include <vector>

#include "internal.h"
#include "unpermute.h"

namespace tl {

constexpr int kGatherThreads = 256;

// A run of top keys as the gather reads it: element e comes from C[src + e]
// and goes to tile offset btree_top_item_off(run, e).
struct GatherRun {
    uint64_t src;
    uint32_t off0, mult, rb, pad;
};

struct GatherShared {
    GatherRun runs[kMaxTopRuns];
    uint32_t cum[kMaxTopRuns + 1];
    uint32_t nslots;
    Regime reg;
};

// Warp 0: the tile's runs of top keys, one lane per slot, and their prefix sums.
__device__ __forceinline__ void gather_runs_warp(const BtreeStream &S, uint64_t p0, uint64_t p1, GatherShared &gs) {
    const uint32_t lane = threadIdx.x;
    TopGroup G0{}, G1{};
    const int ng = btree_stream_groups(S, p0, p1, G0, G1);
    const uint32_t h = S.g.h, nslots = (uint32_t)ng * h;
    uint32_t carry = 0;
    for (uint32_t s0 = 0; s0 < nslots; s0 += 32) {
        const uint32_t sl = s0 + lane;
        TopRun run{};
        if (sl < nslots) run = btree_group_run(S, sl < h ? G0 : G1, sl < h ? sl : sl - h, p0 >> S.tile_shift);
        uint32_t incl = run.cnt;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, d);
            if (lane >= (uint32_t)d) incl += y;
        }
        if (sl < nslots) {
            gs.runs[sl] = GatherRun{run.dest0, run.off0, run.mult, run.rb, 0};
            gs.cum[sl] = carry + incl - run.cnt;
        }
        carry += __shfl_sync(0xFFFFFFFFu, incl, 31);
    }
    if (lane == 0) {
        gs.cum[nslots] = carry;
        gs.nslots = nslots;
    }
}

// B-tree / BST: sorted tile k gathered from the copy C of the layout.
// The B-tree gather's tile slot of sorted offset o: one padding key after
// every 32, so the top-tree keys written at stride 2^(k+1) (the BST's levels)
// spread over the banks (a stride of 4 to 32 keys: 2 to 4 wavefronts a warp
// instead of 8 to 32), while the final read of consecutive offsets stays
// conflict-free.
__device__ __forceinline__ uint32_t gskew(uint32_t o) { return o + (o >> 5); }

template <typename K>
__global__ void __launch_bounds__(kGatherThreads, 6)
btree_gather_kernel(K *__restrict__ A, const K *__restrict__ C, const __grid_constant__ BtreeStream S) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    K *sm = tile_smem<K>(smem_raw);
    __shared__ GatherShared gs;
    for (uint64_t k = blockIdx.x; k < S.ntiles; k += gridDim.x) {
        uint64_t p0, p1;
        btree_tile(S, k, p0, p1);
        const uint32_t cnt = (uint32_t)(p1 - p0);
        if (threadIdx.x < 32)
            gather_runs_warp(S, p0, p1, gs);
        else if (threadIdx.x == 32)
            gs.reg = btree_stream_regime(S, p0, p1);
        __syncthreads();
        const Regime &R = gs.reg;
        if (R.kind == 0) {
            for (uint64_t x = p0 + threadIdx.x; x < p1; x += blockDim.x)
                if (!btree_is_top(S, x)) sm[gskew((uint32_t)(x - p0))] = C[btree_pos(S.g, S.fd, x)];
        } else if (R.kind == 1) {
            const K *src = C + R.dbase;
            const uint32_t d = S.fd32.d, r0 = R.r0, skip = R.skip;
#pragma unroll 4
            for (uint32_t o = threadIdx.x; o < cnt; o += blockDim.x) {
                const uint32_t v = r0 + o;
                const uint32_t ql = S.fd32.div(v);
                if (v - ql * d != skip) sm[gskew(o)] = src[v - ql];
            }
        }
        // the tile's top keys, four items a thread at a time: their loads in
        // flight together
        const uint32_t total = gs.cum[gs.nslots];
        uint32_t r = 0;
        for (uint32_t g0 = threadIdx.x; g0 < total; g0 += 4 * blockDim.x) {
            K v[4];
            uint32_t off[4];
#pragma unroll
            for (int t = 0; t < 4; ++t) {
                const uint32_t gi = g0 + t * blockDim.x;
                if (gi < total) {
                    while (gi >= gs.cum[r + 1]) ++r;
                    const GatherRun run = gs.runs[r];
                    const uint32_t e = gi - gs.cum[r];
                    off[t] = btree_top_item_off(S, run, e);
                    v[t] = C[run.src + e];
                }
            }
#pragma unroll
            for (int t = 0; t < 4; ++t)
                if (g0 + t * blockDim.x < total) sm[gskew(off[t])] = v[t];
        }
        __syncthreads();
        for (uint32_t o = threadIdx.x; o < cnt; o += blockDim.x) A[p0 + o] = sm[gskew(o)];
        __syncthreads();  // before the next tile reuses the buffer and the runs
    }
}

// mvEB / standard vEB: sorted tile k gathered unit by unit (a unit's positions
// are contiguous in the layout; its separator, and the keys of a region without
// units, are single keys).
// 4 blocks an SM (48 registers): two units' loads a lane in flight without
// spills; measured on B200, 2^30 - 1 u32 keys, reverse 3.36 ms against 3.82 at
// 6 blocks (spilling) and 3.60 with one unit at a time
template <typename K>
__global__ void __launch_bounds__(kGatherThreads, 4)
veb_gather_kernel(K *__restrict__ A, const K *__restrict__ C, const __grid_constant__ MvebParams prm) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    K *sm = tile_smem<K>(smem_raw);
    __shared__ unsigned char s_inv[256];
    const MvebPlan &P = prm.plan;
    const bool modified = P.modified != 0;
    int loaded_U = -1;
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    for (uint64_t k = blockIdx.x; k < P.total_tiles; k += gridDim.x) {
        int ri;
        uint64_t p0, p1;
        mveb_tile(P, k, ri, p0, p1);
        const MvebRegion &R = P.reg[ri];
        if ((int)R.U != loaded_U && R.U) {  // block-uniform
            const unsigned char *src = prm.inv + unit_table_off(R.U);
            for (uint32_t q = threadIdx.x; q < (1u << R.U) - 1; q += blockDim.x) s_inv[q] = src[q];
            loaded_U = R.U;
            __syncthreads();
        }
        const uint32_t cnt = (uint32_t)(p1 - p0);
        if (R.U == 0) {
            for (uint64_t x = p0 + threadIdx.x; x < p1; x += blockDim.x) sm[x - p0] = C[veb_pos(P.n, x, modified)];
        } else {
            const uint32_t U = R.U;
            const uint64_t u = (1ull << U) - 1;
            uint64_t g0, g1;
            mveb_tile_groups(R, p0, p1, g0, g1);
            // the separators (each a position search of its own): a thread per unit
            for (uint64_t gi = g0 + threadIdx.x; gi < g1; gi += blockDim.x) {
                const uint64_t first = R.src + (gi << U);
                if (first + u < R.src + R.len) sm[first - p0 + u] = C[veb_pos(P.n, first + u, modified)];
            }
            // the units' bodies: a warp per unit, contiguous reads; a warp's units
            // in batches of 32, their positions lane-parallel
            for (uint64_t gb = g0 + warp; gb < g1; gb += 32ull * nwarps) {
                const uint64_t gl = gb + (uint64_t)lane * nwarps;
                const uint64_t my_dst = gl < g1 ? mveb_unit_dst(R, gl) : 0;
                const uint32_t nb = (uint32_t)min((uint64_t)32, (g1 - gb + nwarps - 1) / nwarps);
                for (uint32_t j = 0; j < nb; j += 2) {
                    // two units' at most 255 keys each (U <= 8): a lane issues
                    // all its loads before storing any (a loop that stored each
                    // load waited for them one at a time)
                    const uint32_t j1 = j + 1 < nb ? j + 1 : j;
                    const uint64_t dst0 = __shfl_sync(0xFFFFFFFFu, my_dst, j);
                    const uint64_t dst1 = __shfl_sync(0xFFFFFFFFu, my_dst, j1);
                    const uint32_t o0 = (uint32_t)(R.src + ((gb + (uint64_t)j * nwarps) << U) - p0);
                    const uint32_t o1 = (uint32_t)(R.src + ((gb + (uint64_t)j1 * nwarps) << U) - p0);
                    const uint32_t u1 = j1 != j ? (uint32_t)u : 0u;
                    K v0[8], v1[8];
#pragma unroll
                    for (int jj = 0; jj < 8; ++jj) {
                        const uint32_t q = lane + 32u * jj;
                        if (q < u) v0[jj] = C[dst0 + q];
                        if (q < u1) v1[jj] = C[dst1 + q];
                    }
#pragma unroll
                    for (int jj = 0; jj < 8; ++jj) {
                        const uint32_t q = lane + 32u * jj;
                        if (q < u) sm[o0 + s_inv[q]] = v0[jj];
                        if (q < u1) sm[o1 + s_inv[q]] = v1[jj];
                    }
                }
            }
        }
        __syncthreads();
        for (uint32_t o = threadIdx.x; o < cnt; o += blockDim.x) A[p0 + o] = sm[o];
        __syncthreads();
    }
}

// ---------------------------------------------------------------- host side
static inline uint64_t align256(uint64_t x) { return (x + 255) / 256 * 256; }

int unpermute_workspace_bytes(int layout, uint64_t n, uint64_t b, uint32_t key_bytes, uint64_t *bytes) {
    if (!bytes) return TL_ERROR_INVALID_VALUE;
    PermuteGeometry geo;
    const int rc = permute_geometry(layout, n, b, key_bytes, geo);
    if (rc) return rc;
    *bytes = align256(n * key_bytes);
    return TL_SUCCESS;
}

static int g_gather_sms = 0;
static std::once_flag g_gather_once;

template <typename K>
static int launch_unpermute(const PermuteGeometry &geo, K *A, const K *C, cudaStream_t st) {
    std::call_once(g_gather_once, [] {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&g_gather_sms, cudaDevAttrMultiProcessorCount, dev);
        if (g_gather_sms <= 0) g_gather_sms = 148;
    });
    const size_t smem = (size_t)geo.tile_keys * sizeof(K) + kTileSmemSlack;
    int per_sm = 0;
    if (is_veb_layout(geo.layout)) {
        auto kern = veb_gather_kernel<K>;
        TL_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        TL_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kGatherThreads, smem));
        const uint64_t grid = std::min<uint64_t>((uint64_t)std::max(per_sm, 1) * g_gather_sms, geo.ntiles);
        kern<<<(unsigned)grid, kGatherThreads, smem, st>>>(A, C, geo.mp);
    } else {
        auto kern = btree_gather_kernel<K>;
        const size_t smem_b = smem + (geo.tile_keys / 32 + 1) * sizeof(K);  // gskew's padding keys
        TL_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_b));
        TL_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kGatherThreads, smem_b));
        const uint64_t grid = std::min<uint64_t>((uint64_t)std::max(per_sm, 1) * g_gather_sms, geo.ntiles);
        kern<<<(unsigned)grid, kGatherThreads, smem_b, st>>>(A, C, geo.bs);
    }
    TL_CUDA_TRY(cudaGetLastError());
    return TL_SUCCESS;
}

// The geometry with the B-tree read as under the right-to-left schedule: the
// last level as bulk keys (from position ni on) and every top-tree level as runs.
static int gather_geometry(int layout, uint64_t n, uint64_t b, uint32_t key_bytes, PermuteGeometry &geo) {
    const int rc = permute_geometry(layout, n, b, key_bytes, geo);
    if (rc) return rc;
    geo.bs.plan = PLAN_R;
    return TL_SUCCESS;
}

int unpermute(int layout, void *dev_A, uint64_t n, uint64_t b, uint32_t key_bytes, void *dev_ws, uint64_t ws_bytes,
              cudaStream_t st, float *ms) {
    if (n > 0 && !dev_A) return TL_ERROR_INVALID_VALUE;
    if (reinterpret_cast<uintptr_t>(dev_A) % (key_bytes ? key_bytes : 1)) return TL_ERROR_INVALID_VALUE;
    if (dev_ws && reinterpret_cast<uintptr_t>(dev_ws) % 256) return TL_ERROR_INVALID_VALUE;
    PermuteGeometry geo;
    int rc = gather_geometry(layout, n, b, key_bytes, geo);
    if (rc) return rc;
    if (n <= 1) {
        if (ms) *ms = 0.f;
        return TL_SUCCESS;
    }
    const uint64_t need = align256(n * key_bytes);
    if (dev_ws && ws_bytes < need) return TL_ERROR_WORKSPACE_TOO_SMALL;
    EventTimer timer(ms != nullptr, st);
    char *ws = static_cast<char *>(dev_ws);
    bool owned = false;
    bool pooled = false;
    if (!ws) {
        ws = static_cast<char *>(workspace_acquire(need));
        if (ws) {
            owned = true;
        } else {  // the cache could not help: a stream-ordered allocation
            keep_pool_memory();
            if (cudaMallocAsync(reinterpret_cast<void **>(&ws), need, st) != cudaSuccess) {
                record_cuda_error(cudaGetLastError());
                return TL_ERROR_OUT_OF_MEMORY;
            }
            owned = pooled = true;
        }
    }
    timer.start();
    rc = TL_SUCCESS;
    if (cudaMemcpyAsync(ws, dev_A, n * key_bytes, cudaMemcpyDeviceToDevice, st) != cudaSuccess) {
        record_cuda_error(cudaGetLastError());
        rc = TL_ERROR_CUDA;
    }
    if (rc == TL_SUCCESS)
        rc = key_bytes == 8 ? launch_unpermute<uint64_t>(geo, static_cast<uint64_t *>(dev_A),
                                                         reinterpret_cast<const uint64_t *>(ws), st)
                            : launch_unpermute<uint32_t>(geo, static_cast<uint32_t *>(dev_A),
                                                         reinterpret_cast<const uint32_t *>(ws), st);
    timer.stop();
    if (owned && pooled) cudaFreeAsync(ws, st);
    if (rc == TL_SUCCESS) rc = sync_and_check(st);
    if (owned && !pooled) {
        if (rc != TL_SUCCESS) cudaStreamSynchronize(st);  // nothing of this call may still use it
        workspace_release(ws);
    }
    if (rc == TL_SUCCESS && ms) *ms = timer.elapsed();
    return rc;
}

// Host replay of the gather with the kernels' per-tile helpers (test hook).
int emulate_unpermute(int layout, uint64_t n, uint64_t b, uint64_t *A) {
    if (n > 0 && !A) return TL_ERROR_INVALID_VALUE;
    PermuteGeometry geo;
    const int rc = gather_geometry(layout, n, b, 8, geo);
    if (rc) return rc;
    if (n <= 1) return TL_SUCCESS;
    const std::vector<uint64_t> C(A, A + n);
    std::vector<uint64_t> tile(geo.tile_keys + 1);
    std::vector<uint8_t> got(n, 0);
    if (is_veb_layout(layout)) {
        const MvebPlan &P = geo.mp.plan;
        const bool modified = P.modified != 0;
        for (uint64_t k = 0; k < P.total_tiles; ++k) {
            int ri;
            uint64_t p0, p1;
            mveb_tile(P, k, ri, p0, p1);
            const MvebRegion &R = P.reg[ri];
            if (R.U == 0) {
                for (uint64_t x = p0; x < p1; ++x) tile[x - p0] = C[veb_pos(n, x, modified)];
            } else {
                const unsigned char *inv = geo.mp.inv + unit_table_off(R.U);
                const uint64_t u = (1ull << R.U) - 1;
                uint64_t g0, g1;
                mveb_tile_groups(R, p0, p1, g0, g1);
                for (uint64_t gi = g0; gi < g1; ++gi) {
                    const uint64_t first = R.src + (gi << R.U), dst = mveb_unit_dst(R, gi);
                    if (first < p0 || first + u > p0 + geo.tile_keys) return TL_ERROR_UNSUPPORTED;  // units tile the tile
                    for (uint64_t q = 0; q < u; ++q) tile[first - p0 + inv[q]] = C[dst + q];
                    if (first + u < R.src + R.len) tile[first - p0 + u] = C[veb_pos(n, first + u, modified)];
                }
            }
            for (uint64_t x = p0; x < p1; ++x) {
                A[x] = tile[x - p0];
                ++got[x];
            }
        }
    } else {
        const BtreeStream &S = geo.bs;
        for (uint64_t k = 0; k < S.ntiles; ++k) {
            uint64_t p0, p1;
            btree_tile(S, k, p0, p1);
            const uint32_t cnt = (uint32_t)(p1 - p0);
            const Regime R = btree_stream_regime(S, p0, p1);
            if (R.kind == 0) {
                for (uint64_t x = p0; x < p1; ++x)
                    if (!btree_is_top(S, x)) tile[x - p0] = C[btree_pos(S.g, S.fd, x)];
            } else if (R.kind == 1) {
                for (uint32_t o = 0; o < cnt; ++o) {
                    uint64_t idx;
                    if (btree_regime_bulk(S, R, o, idx)) tile[o] = C[idx];
                }
            }
            TopGroup G0{}, G1{};
            const int ng = btree_stream_groups(S, p0, p1, G0, G1);
            for (int gq = 0; gq < ng; ++gq)
                for (uint32_t lv = 0; lv < S.g.h; ++lv) {
                    const TopRun run = btree_group_run(S, gq ? G1 : G0, lv, k);
                    for (uint32_t e = 0; e < run.cnt; ++e) tile[btree_top_item_off(S, run, e)] = C[run.dest0 + e];
                }
            for (uint64_t x = p0; x < p1; ++x) {
                A[x] = tile[x - p0];
                ++got[x];
            }
        }
    }
    for (uint64_t x = 0; x < n; ++x)
        if (got[x] != 1) return TL_ERROR_UNSUPPORTED;
    return TL_SUCCESS;
}

}  // namespace tl
