// In-place permutations sorted -> {B-tree, BST, mvEB} for sm_100a.
//
// Every layout is a pure index permutation with the same two-part structure:
// most keys belong to "bulk" runs (the leaf level of a B-tree, the bottom-level
// subtrees of an mvEB) that land at a position >= their source position, and a
// minority (the separators above them) land further left.  The permutation is
// therefore done in two kernels instead of the reference's chain of cycle-leader
// and reversal launches:
//
//  1. stream: one pass over the array, one tile per ticket.  A tile is read
//     into shared memory, flagged as read, and its bulk keys are stored
//     straight to their final positions once the tiles under those positions
//     have been read.  The other keys go to a scratch buffer.
//  2. B-tree: a copy of the scratch (indexed by final position) into place,
//     or under the ordered-tile schedule the fix pass over the tiles that
//     received scratch keys; mvEB: a scatter of the scratch slots to their
//     final positions.  Every destination is free by then.
//
// DRAM traffic is 2*n*w for the stream plus 2*w per scratch key: 6-20 % of the
// keys of a B-tree or BST under the ordered schedule, about n/2^8 for an mvEB.
#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <vector>

#include "btree_order.h"
#include "btree_plan.cuh"
#include "bulk.cuh"
#include "geometry.cuh"
#include "internal.h"
#include "mveb_plan.cuh"
#include "unpermute.h"
#include "stream.cuh"

namespace tl {

constexpr int kStreamThreads = 256;
constexpr int kStreamBlocksPerSM = 6;  // what shared memory allows with 32 KB tiles
constexpr uint32_t kUnitMaxLevels = 8;

template <typename K>
constexpr uint64_t stream_tile_keys() {
    return 32768 / sizeof(K);
}

static inline uint64_t align_up(uint64_t x, uint64_t a) { return (x + a - 1) / a * a; }

// kBst: the instance for b = 1 (see btree_stream_tile's kRunRegs).
template <typename K, bool kBst = false>
__global__ void __launch_bounds__(kStreamThreads, kStreamBlocksPerSM)
btree_stream_kernel(K *__restrict__ A, K *__restrict__ scr, const __grid_constant__ BtreeStream S, Ctrl *ctrl,
                    WaitCfg wc, unsigned int *flags) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    K *sm = tile_smem<K>(smem_raw);
    __shared__ unsigned long long s_ticket;
    __shared__ TileShared ts;
    TicketPipe tp;
    for (unsigned long long t = ticket_first(ctrl, &s_ticket); t < S.ntiles; t = ticket_advance(tp, &s_ticket)) {
        ticket_claim(ctrl, tp);
        btree_stream_tile<K, kBst>(S, A, scr, flags, ctrl, wc, btree_tile_of_ticket(S, t), sm, ts);
    }
}

// Second pass of a B-tree permutation: the scratch ranges to their final
// positions, a plain copy (scratch is indexed by final position) through the
// bulk-copy engine.
template <typename K>
__global__ void __launch_bounds__(32)
btree_copy_kernel(K *__restrict__ A, const K *__restrict__ scr, const __grid_constant__ BulkPlan P, Ctrl *ctrl) {
    extern __shared__ __align__(128) unsigned char stage[];
    __shared__ __align__(8) uint64_t bars[kBulkStages];
    bulk_copy_plan(A, scr, P, stage, bars, ctrl);
}

// Second pass of a plan-O B-tree permutation for the scratch keys outside the
// whole-tile ranges: the host-listed copies, a warp per copy.
template <typename K>
__global__ void __launch_bounds__(kScatterThreads)
btree_fix_kernel(K *__restrict__ A, const K *__restrict__ scr, const FixSeg *__restrict__ segs, uint64_t nsegs) {
    const uint64_t w = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t i = w; i < nsegs; i += nw) {
        const uint64_t dl = __ldg(reinterpret_cast<const unsigned long long *>(&segs[i].dst_len));
        const uint64_t src = __ldg(reinterpret_cast<const unsigned long long *>(&segs[i].src));
        warp_copy_keys(A + (dl & kSegDstMask), scr + src, 0, (uint32_t)(dl >> 48));
    }
}

// One copy range for the bulk engine: its 16-byte-aligned interior in
// kBulkChunk pieces, its ragged keys apart.  The scratch shares A's offset
// within 16 bytes at both range bases, so the interiors line up.
template <typename K>
static int add_bulk_range(const K *A, const K *scr, const CopyRange &r, BulkPlan &P) {
    if (P.nr == kMaxBulkRanges) return TL_ERROR_UNSUPPORTED;
    const uintptr_t da = reinterpret_cast<uintptr_t>(A + r.dst), sa = reinterpret_cast<uintptr_t>(scr + r.src);
    if ((da ^ sa) & 15) return TL_ERROR_INVALID_VALUE;
    BulkRange R{};
    R.key_dst = r.dst;
    R.key_src = r.src;
    R.len = r.len;
    const uint64_t head = std::min<uint64_t>(((16 - (da & 15)) & 15) / sizeof(K), r.len);
    const uint64_t body = ((r.len - head) * sizeof(K)) & ~15ull;
    R.head = (uint32_t)head;
    R.tail = (uint32_t)(r.len - head - body / sizeof(K));
    R.dst = (r.dst + head) * sizeof(K);
    R.src = (r.src + head) * sizeof(K);
    R.bytes = body;
    R.chunk0 = P.nchunks;
    P.nchunks += (body + kBulkChunk - 1) / kBulkChunk;
    P.r[P.nr++] = R;
    return TL_SUCCESS;
}

// The copy ranges of a plan: per level (plans R, L), or the runs of whole
// scratch tiles (plan O: tiles [x, y) from scratch slot z on).
template <typename K>
static int make_bulk_plan(const BtreeStream &S, const OrderTables &ot, const K *A, const K *scr, BulkPlan &P) {
    P.nr = 0;
    P.nchunks = 0;
    if (S.plan == PLAN_O) {
        for (uint64_t i = 0; i < ot.nranges; ++i) {
            const uint64_t u0 = ot.ranges[i].x, u1 = ot.ranges[i].y;
            const uint64_t d0 = u0 << S.tile_shift, d1 = std::min<uint64_t>(u1 << S.tile_shift, S.g.n);
            const uint64_t s0 = (uint64_t)ot.ranges[i].z << S.tile_shift;  // host data: S.tab may be device memory
            const int rc = add_bulk_range(A, scr, CopyRange{d0, s0, d1 - d0}, P);
            if (rc) return rc;
        }
        return TL_SUCCESS;
    }
    for (int j = 0; j < btree_copy_range_count(S); ++j) {
        CopyRange r;
        if (!btree_copy_range(S, j, r)) continue;
        const int rc = add_bulk_range(A, scr, r, P);
        if (rc) return rc;
    }
    return TL_SUCCESS;
}

// ---------------------------------------------------------------- mvEB stream
template <typename K>
__global__ void __launch_bounds__(kStreamThreads, kStreamBlocksPerSM)
mveb_stream_kernel(K *__restrict__ A, K *__restrict__ scr, const __grid_constant__ MvebParams prm,
                   Ctrl *ctrl, WaitCfg wc, unsigned int *flags) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    K *sm = reinterpret_cast<K *>(smem_raw);  // see load_tile_issue
    __shared__ unsigned long long s_ticket;
    __shared__ int s_ok;
    __shared__ unsigned char s_inv[256];
    const MvebPlan &P = prm.plan;
    const uint64_t ntiles = P.total_tiles;
    int loaded_U = -1;
    uint32_t inv_pk[2] = {0, 0};  // this lane's entries of the unit table (see below)
    const uint32_t lane = threadIdx.x & 31;
    // The next ticket is claimed as the tile ends, not as it starts: a tile's
    // stores wait for the tiles just right of it, claimed just before it, and a
    // ticket held through a whole tile made those waits long (measured on B200,
    // 2^30 - 1 u32 keys: stalled waits 8.2e4 -> 4.8e4, 1.83 -> 1.81 ms).
    TicketPipe tp;
    for (unsigned long long t = ticket_first(ctrl, &s_ticket); t < ntiles; t = ticket_advance(tp, &s_ticket)) {
        const uint64_t k = ntiles - 1 - t;
        int ri;
        uint64_t p0, p1;
        mveb_tile(P, k, ri, p0, p1);
        const MvebRegion &R = P.reg[ri];
        if ((int)R.U != loaded_U && R.U) {  // block-uniform: unit tables for this height
            const unsigned char *src = prm.inv + unit_table_off(R.U);
            __syncthreads();  // every lane has its packed entries of the previous table
            for (uint32_t q = threadIdx.x; q < (1u << R.U) - 1; q += blockDim.x) s_inv[q] = src[q];
            __syncthreads();
            // each lane's entries q = lane + 32 j (j < 8), four per register
            inv_pk[0] = inv_pk[1] = 0;
            const uint32_t uu = (1u << R.U) - 1;
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const uint32_t q = lane + 32u * j;
                if (q < uu) inv_pk[j >> 2] |= (uint32_t)s_inv[q] << (8 * (j & 3));
            }
            loaded_U = R.U;
        }
        if (threadIdx.x == 0) s_ok = 1;  // the previous tile's readers are past the ticket barrier
        const uint64_t base = load_tile<16>(A, p0, p1, sm);
        publish_read(&flags[k], wc);
        if (R.U == 0) {
            for (uint64_t x = p0 + threadIdx.x; x < p1; x += blockDim.x)
                scr[R.slot_base + (x - R.src)] = sm[x - base];
            ticket_claim(ctrl, tp);
            continue;
        }
        uint64_t k_lo, k_hi;
        if (mveb_tile_wait(P, R, p0, p1, k_lo, k_hi)) {
            for (uint64_t f = k_lo + threadIdx.x; f <= k_hi; f += blockDim.x)
                if (!wait_flag(&flags[f], wc.wait_value, ctrl, wc)) s_ok = 0;
            __syncthreads();
            if (!s_ok) {
                ticket_claim(ctrl, tp);
                continue;
            }
        }
        const uint32_t U = R.U;
        const uint64_t u = (1ull << U) - 1;
        uint64_t g0, g1;
        mveb_tile_groups(R, p0, p1, g0, g1);
        const uint32_t warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
        // a warp's units in batches of 32: their destinations lane-parallel, one
        // unit per lane, then each unit's keys by the whole warp
        for (uint64_t gb = g0 + warp; gb < g1; gb += 32ull * nwarps) {
            const uint64_t gl = gb + (uint64_t)lane * nwarps;
            const uint64_t my_dst = gl < g1 ? mveb_unit_dst(R, gl) : 0;
            const uint32_t nb = (uint32_t)std::min<uint64_t>(32, (g1 - gb + nwarps - 1) / nwarps);
            for (uint32_t j = 0; j < nb; ++j) {
                const uint64_t gi = gb + (uint64_t)j * nwarps;
                const uint64_t dst = __shfl_sync(0xFFFFFFFFu, my_dst, j);
                const uint32_t gsrc = (uint32_t)(R.src + (gi << U) - base);
                K *d = A + dst + lane;
                const K *g = sm + gsrc;
#pragma unroll
                for (int jj = 0; jj < 8; ++jj)
                    if (lane + 32u * jj < (uint32_t)u) d[32 * jj] = g[(inv_pk[jj >> 2] >> (8 * (jj & 3))) & 0xFFu];
                if (lane == 0 && R.src + (gi << U) + u < R.src + R.len)
                    scr[R.slot_base + gi] = sm[gsrc + u];
            }
        }
        ticket_claim(ctrl, tp);
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
            if (rank != ~0ull) A[veb_pos(P.n, rank, P.modified != 0)] = v[u];
        }
    }
    for (; s < P.total_slots; s += stride) {
        const uint64_t rank = mveb_slot_rank(P, s);
        if (rank != ~0ull) A[veb_pos(P.n, rank, P.modified != 0)] = scr[s];
    }
}

// ---------------------------------------------------------------- host side
struct PermutePlan {
    int layout = 0;
    uint32_t key_bytes = 8;
    uint64_t n = 0, b = 1;
    uint64_t tile_keys = 0, ntiles = 0, scratch_keys = 0;
    bool ordered = false;  // B-tree plan O, with these tables (host, then device pointers)
    OrderTables ot;
    BtreeStream bs;
    MvebParams mp;
    uint64_t off_flags = 0, off_ctrl = 0, bytes = 0;
};

// When a B-tree permutation takes plan O: ORDER_AUTO from kOrderMinTiles tiles
// up (below that a tile order has too few tiles to pay for its second pass),
// for a BST from kOrderMinTilesBst (measured on B200, u64 keys: at 2^20 - 1
// the fixed schedule takes 34 us against 42, its second pass one launch
// instead of two; at 2^26 - 1 they tie, 0.289 against 0.290 ms), ORDER_ALWAYS
// whenever there is a top tree and more than one tile (host replay).
enum OrderMode { ORDER_NEVER = 0, ORDER_AUTO = 1, ORDER_ALWAYS = 2 };
constexpr uint64_t kOrderMinTiles = 64;
constexpr uint64_t kOrderMinTilesBst = 16384;
// tl_debug_set_schedule: 1 = ORDER_AUTO acts as ORDER_NEVER; 2 = batched plans
// order every instance that can take the ordered schedule
static std::atomic<int> g_schedule_mode{0};

void set_schedule_mode(int mode) { g_schedule_mode = mode; }
bool fixed_schedule_only() { return g_schedule_mode == 1; }
bool ordered_schedule_forced() { return g_schedule_mode == 2; }

// Plan O's tables come from the library's cache unless `tables` are given.
// Whether a B-tree / BST plan takes the ordered-tile schedule in order_mode.
static bool order_wanted(const PermutePlan &pl, int order_mode) {
    return pl.bs.g.h >= 1 && pl.ntiles >= 2 &&
           (order_mode == ORDER_ALWAYS ||
            (order_mode == ORDER_AUTO && pl.ntiles >= (pl.b == 1 ? kOrderMinTilesBst : kOrderMinTiles) &&
             !fixed_schedule_only()));
}

static int make_plan(int layout, uint64_t n, uint64_t b, uint32_t key_bytes, PermutePlan &pl,
                     int order_mode = ORDER_AUTO, const OrderTables *tables = nullptr) {
    if (key_bytes != 4 && key_bytes != 8) return TL_ERROR_INVALID_VALUE;
    if (layout == TL_LAYOUT_BST) b = 1;
    if (layout == TL_LAYOUT_BTREE && b == 0) return TL_ERROR_INVALID_VALUE;
    if (layout < TL_LAYOUT_BST || layout > TL_LAYOUT_VEB) return TL_ERROR_INVALID_VALUE;
    pl.layout = layout;
    pl.key_bytes = key_bytes;
    pl.n = n;
    pl.b = b;
    pl.tile_keys = 32768 / key_bytes;
    if (is_veb_layout(layout)) {
        if (n >= (1ull << 62)) return TL_ERROR_UNSUPPORTED;
        pl.mp.plan = make_mveb_plan(n, kUnitMaxLevels, pl.tile_keys, layout == TL_LAYOUT_MVEB);
        fill_unit_tables(pl.mp);
        pl.ntiles = pl.mp.plan.total_tiles;
        pl.scratch_keys = pl.mp.plan.total_slots;
    } else {
        if (b >= (1ull << 31)) return TL_ERROR_UNSUPPORTED;
        pl.bs.g = make_btree_geom(n, b);
        // per-level tables and 32-bit tile indices of the wait lists
        if (pl.bs.g.h > (uint32_t)kMaxTopLevels || n / pl.tile_keys >= (1ull << 32)) return TL_ERROR_UNSUPPORTED;
        pl.bs.fd = FastDiv64(b + 1);
        pl.bs.fd32 = FastDiv32((uint32_t)(b + 1));
        if (b >= 2) {
            pl.bs.fd32b = FastDiv32((uint32_t)b);
            pl.bs.fdb = FastDiv64(b);
        }
        pl.bs.tile_keys = pl.tile_keys;
        pl.bs.tile_shift = (uint32_t)__builtin_ctzll(pl.tile_keys);
        btree_set_pow_divs(pl.bs, make_pow_divs(b));
        pl.ntiles = (n + pl.tile_keys - 1) / pl.tile_keys;
        pl.bs.ntiles = pl.ntiles;
        btree_choose_plan(pl.bs, key_bytes);
        if (order_wanted(pl, order_mode)) {
            if (tables) pl.ot = *tables;
            if (tables || btree_order_host(pl.bs, pl.ot)) {
                btree_set_ordered(pl.bs, pl.ot.tab, pl.ot.order, pl.ot.scratch_tiles);
                pl.ordered = true;
            }
        }
        pl.scratch_keys = pl.bs.nscratch;
    }
    // + 16 bytes: the scratch starts at the array's own offset within 16 bytes
    pl.off_flags = align_up(pl.scratch_keys * key_bytes + 16, 256);
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

static std::atomic<int> g_last_launches{0};  // kernels the last permutation launched (profiling hook)

int last_permute_launches() { return g_last_launches; }

template <typename K>
static int launch_permute_k(const PermutePlan &pl, K *A, char *ws, cudaStream_t st, EventTimer &timer, int &nl);

template <typename K>
static int launch_permute(const PermutePlan &pl, K *A, char *ws, cudaStream_t st, EventTimer &timer) {
    int nl = 0;
    const int rc = launch_permute_k(pl, A, ws, st, timer, nl);
    g_last_launches = nl;
    return rc;
}

template <typename K>
static int launch_permute_k(const PermutePlan &pl, K *A, char *ws, cudaStream_t st, EventTimer &timer, int &nl) {
    // the scratch shares A's offset within 16 bytes, so the copy pass vectorises
    K *scr = reinterpret_cast<K *>(ws + (reinterpret_cast<uintptr_t>(A) & 15));
    unsigned int *flags = reinterpret_cast<unsigned int *>(ws + pl.off_flags);
    Ctrl *ctrl = reinterpret_cast<Ctrl *>(ws + pl.off_ctrl);
    WaitCfg wc;
    wc.flag_value = 1;
    wc.wait_value = debug_force_timeout() ? 0xFFFFFFFFu : 1u;  // forced: no tile ever publishes it
    wc.spin_limit = debug_spin_limit();
    // flags and control block are contiguous: one stream-ordered memset clears both
    TL_CUDA_TRY(cudaMemsetAsync(flags, 0, pl.bytes - pl.off_flags, st));
    const size_t smem = (size_t)pl.tile_keys * sizeof(K) + kTileSmemSlack;
    const int smx = sm_count();
    if (is_veb_layout(pl.layout)) {
        auto kern = mveb_stream_kernel<K>;
        TL_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        int per_sm = 0;
        TL_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kStreamThreads, smem));
        uint64_t grid = std::min<uint64_t>((uint64_t)std::max(per_sm, 1) * smx, std::max<uint64_t>(pl.ntiles, 1));
        if (pl.ntiles) kern<<<(unsigned)grid, kStreamThreads, smem, st>>>(A, scr, pl.mp, ctrl, wc, flags), ++nl;
        TL_CUDA_TRY(cudaGetLastError());
        timer.mid();
        if (pl.scratch_keys) {
            int sper = 0;
            TL_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&sper, mveb_scatter_kernel<K>,
                                                                      kScatterThreads, 0));
            uint64_t sg = std::min<uint64_t>((pl.scratch_keys + kScatterThreads - 1) / kScatterThreads,
                                             (uint64_t)std::max(sper, 1) * smx);
            mveb_scatter_kernel<K><<<(unsigned)sg, kScatterThreads, 0, st>>>(A, scr, pl.mp);
            ++nl;
            TL_CUDA_TRY(cudaGetLastError());
        }
    } else {
        auto kern = pl.bs.g.b == 1 ? btree_stream_kernel<K, true> : btree_stream_kernel<K, false>;
        TL_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        int per_sm = 0;
        TL_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kStreamThreads, smem));
        uint64_t grid = std::min<uint64_t>((uint64_t)std::max(per_sm, 1) * smx, std::max<uint64_t>(pl.ntiles, 1));
        if (pl.ntiles) kern<<<(unsigned)grid, kStreamThreads, smem, st>>>(A, scr, pl.bs, ctrl, wc, flags), ++nl;
        TL_CUDA_TRY(cudaGetLastError());
        timer.mid();
        if (pl.ordered && pl.ot.nsegs) {
            int fper = 0;
            TL_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&fper, btree_fix_kernel<K>, kScatterThreads, 0));
            const uint64_t fg = std::min<uint64_t>((pl.ot.nsegs * 32 + kScatterThreads - 1) / kScatterThreads,
                                                   (uint64_t)std::max(fper, 1) * smx);
            btree_fix_kernel<K><<<(unsigned)fg, kScatterThreads, 0, st>>>(A, scr, pl.ot.segs, pl.ot.nsegs);
            ++nl;
            TL_CUDA_TRY(cudaGetLastError());
        }
        BulkPlan bp;
        int rc = make_bulk_plan(pl.bs, pl.ot, A, scr, bp);
        if (rc) return rc;
        if (bp.nr) {
            // one warp per CTA, as many CTAs per SM as the stages' shared memory allows
            const size_t smem = (size_t)kBulkStages * kBulkChunk;
            auto ck = btree_copy_kernel<K>;
            TL_CUDA_TRY(cudaFuncSetAttribute(ck, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            int cper = 0;
            TL_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&cper, ck, 32, smem));
            const uint64_t cg = std::max<uint64_t>(1, std::min<uint64_t>(bp.nchunks, (uint64_t)std::max(cper, 1) * smx));
            ck<<<(unsigned)cg, 32, smem, st>>>(A, scr, bp, ctrl);
            ++nl;
            TL_CUDA_TRY(cudaGetLastError());
        }
    }
    return TL_SUCCESS;
}

int btree_plan_of(uint64_t n, uint64_t b) {
    PermutePlan pl;
    if (make_plan(TL_LAYOUT_BTREE, n, b, 8, pl, ORDER_NEVER)) return -1;
    return pl.bs.plan;
}

template <typename Kern>
static int blocks_per_sm_of(Kern kern, size_t smem) {
    int per_sm = 0;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kStreamThreads, smem) != cudaSuccess)
        return -1;
    return per_sm;
}

// Resident blocks per SM of the stream kernel instance launch_permute_k picks
// for the layout (the BST has its own instance), at the 32 KB tile.
int stream_blocks_per_sm(int layout, uint32_t key_bytes) {
    const size_t smem = 32768 + kTileSmemSlack;
    const bool w8 = key_bytes == 8;
    if (is_veb_layout(layout))
        return w8 ? blocks_per_sm_of(mveb_stream_kernel<uint64_t>, smem)
                  : blocks_per_sm_of(mveb_stream_kernel<uint32_t>, smem);
    if (layout == TL_LAYOUT_BST)
        return w8 ? blocks_per_sm_of(btree_stream_kernel<uint64_t, true>, smem)
                  : blocks_per_sm_of(btree_stream_kernel<uint32_t, true>, smem);
    return w8 ? blocks_per_sm_of(btree_stream_kernel<uint64_t, false>, smem)
              : blocks_per_sm_of(btree_stream_kernel<uint32_t, false>, smem);
}

int permute_geometry(int layout, uint64_t n, uint64_t b, uint32_t key_bytes, PermuteGeometry &geo) {
    PermutePlan pl;
    const int rc = make_plan(layout, n, b, key_bytes, pl, ORDER_NEVER);
    if (rc) return rc;
    geo.layout = pl.layout;
    geo.key_bytes = pl.key_bytes;
    geo.n = pl.n;
    geo.tile_keys = pl.tile_keys;
    geo.ntiles = pl.ntiles;
    geo.bs = pl.bs;
    geo.mp = pl.mp;
    return TL_SUCCESS;
}

int permute_plan_of(int layout, uint64_t n, uint64_t b, uint32_t key_bytes) {
    PermutePlan pl;
    const int rc = make_plan(layout, n, b, key_bytes, pl);
    if (rc) return -rc;
    return is_veb_layout(layout) ? 3 : pl.bs.plan;
}

int permute_scratch_keys(int layout, uint64_t n, uint64_t b, uint32_t key_bytes, uint64_t *keys) {
    if (!keys) return TL_ERROR_INVALID_VALUE;
    PermutePlan pl;
    int rc = make_plan(layout, n, b, key_bytes, pl);
    if (rc) return rc;
    if (is_veb_layout(layout)) {
        *keys = pl.mp.plan.total_slots;
    } else if (pl.ordered) {
        uint64_t c = 0;
        for (uint64_t i = 0; i < pl.ot.nranges; ++i)
            c += std::min<uint64_t>((uint64_t)pl.ot.ranges[i].y << pl.bs.tile_shift, n) -
                 ((uint64_t)pl.ot.ranges[i].x << pl.bs.tile_shift);
        for (uint64_t i = 0; i < pl.ot.nsegs; ++i) c += pl.ot.segs[i].dst_len >> 48;
        *keys = c;
    } else {
        *keys = 0;
        CopyRange r;
        for (int j = 0; j < btree_copy_range_count(pl.bs); ++j)
            if (btree_copy_range(pl.bs, j, r)) *keys += r.len;
    }
    return TL_SUCCESS;
}

// Enough for whichever schedule the call ends up on: the ordered schedule when
// its tables reach the device, else the fixed-direction one (permute() falls
// back to it when the table upload fails), so a workspace of this size is never
// refused.
int permute_workspace_bytes(int layout, uint64_t n, uint64_t b, uint32_t key_bytes, uint64_t *bytes) {
    if (!bytes) return TL_ERROR_INVALID_VALUE;
    PermutePlan pl, fx;
    int rc = make_plan(layout, n, b, key_bytes, pl);
    if (rc) return rc;
    rc = make_plan(layout, n, b, key_bytes, fx, ORDER_NEVER);
    if (rc) return rc;
    *bytes = std::max(pl.bytes, fx.bytes);
    return TL_SUCCESS;
}

int permute_workspace_bytes_fixed(int layout, uint64_t n, uint64_t b, uint32_t key_bytes, uint64_t *bytes) {
    if (!bytes) return TL_ERROR_INVALID_VALUE;
    PermutePlan pl;
    int rc = make_plan(layout, n, b, key_bytes, pl, ORDER_NEVER);
    if (rc) return rc;
    *bytes = pl.bytes;
    return TL_SUCCESS;
}

int permute(int layout, void *dev_A, uint64_t n, uint64_t b, uint32_t key_bytes, void *dev_ws,
            uint64_t ws_bytes, cudaStream_t st, float *ms, float *phase_ms, bool allow_ordered) {
    if (n > 0 && !dev_A) return TL_ERROR_INVALID_VALUE;
    if (reinterpret_cast<uintptr_t>(dev_A) % (key_bytes ? key_bytes : 1)) return TL_ERROR_INVALID_VALUE;
    if (dev_ws && reinterpret_cast<uintptr_t>(dev_ws) % 256) return TL_ERROR_INVALID_VALUE;
    PermutePlan pl;
    if (allow_ordered && n > 1 && !is_veb_layout(layout)) {
        // a geometry not seen before: its ordered-tile tables with kernels on
        // st (make_plan below finds them cached; if this cannot be done it
        // computes them on the host)
        PermutePlan fx;
        if (make_plan(layout, n, b, key_bytes, fx, ORDER_NEVER) == TL_SUCCESS && order_wanted(fx, ORDER_AUTO))
            btree_order_prepare(fx.bs, st);
    }
    int rc = make_plan(layout, n, b, key_bytes, pl, allow_ordered ? ORDER_AUTO : ORDER_NEVER);
    if (rc) return rc;
    if (n <= 1) {
        if (ms) *ms = 0.f;
        return TL_SUCCESS;
    }
    // plan O needs its tile tables on the device and a scratch over every
    // position; without either, the fixed-direction plan
    if (pl.ordered) {
        OrderTables dt;
        if ((dev_ws && ws_bytes < pl.bytes) || !btree_order_device(pl.bs, st, dt)) {
            rc = make_plan(layout, n, b, key_bytes, pl, ORDER_NEVER);
            if (rc) return rc;
        } else {
            pl.ot = dt;
            pl.bs.tab = dt.tab;
            pl.bs.order = dt.order;
        }
    }
    if (dev_ws && ws_bytes < pl.bytes) return TL_ERROR_WORKSPACE_TOO_SMALL;
    EventTimer timer(ms != nullptr || phase_ms != nullptr, st);
    char *ws = static_cast<char *>(dev_ws);
    bool owned = false;
    bool pooled = false;
    if (!ws) {
        ws = static_cast<char *>(workspace_acquire(pl.bytes));
        if (ws) {
            owned = true;
        } else {  // the cache could not help: a stream-ordered allocation
            keep_pool_memory();
            if (cudaMallocAsync(reinterpret_cast<void **>(&ws), pl.bytes, st) != cudaSuccess) {
                record_cuda_error(cudaGetLastError());
                return TL_ERROR_OUT_OF_MEMORY;
            }
            owned = pooled = true;
        }
    }
    timer.start();
    rc = key_bytes == 8 ? launch_permute<uint64_t>(pl, static_cast<uint64_t *>(dev_A), ws, st, timer)
                        : launch_permute<uint32_t>(pl, static_cast<uint32_t *>(dev_A), ws, st, timer);
    timer.stop();
    unsigned int err = 0;
    if (rc == TL_SUCCESS) {
        Ctrl *ctrl = reinterpret_cast<Ctrl *>(ws + pl.off_ctrl);
        rc = read_error_word(&ctrl->error, &err, st);
        if (rc == TL_SUCCESS) record_wait_stats(ctrl, st);
    }
    if (owned && pooled) cudaFreeAsync(ws, st);
    if (rc == TL_SUCCESS) rc = sync_and_check(st);
    if (owned && !pooled) {
        if (rc != TL_SUCCESS) cudaStreamSynchronize(st);  // nothing of this call may still use it
        workspace_release(ws);
    }
    // a bounded wait expired, or (never expected) the ordered schedule found a
    // scratch store without scratch and skipped it
    if (rc == TL_SUCCESS && err) rc = (err & (1u << TL_ERROR_TIMEOUT)) ? TL_ERROR_TIMEOUT : TL_ERROR_UNSUPPORTED;
    if (rc == TL_SUCCESS && ms) *ms = timer.elapsed();
    if (rc == TL_SUCCESS && phase_ms) timer.elapsed_split(&phase_ms[0], &phase_ms[1]);
    return rc;
}

// Test hook: the ordered-tile tables of a geometry computed on the host and
// with the per-tile kernels on st, uncached, compared entry by entry.  1 equal,
// 0 different, < 0 a status (the geometry takes no ordered tables, or the
// kernels could not run).
int debug_order_tables_match(int layout, uint64_t n, uint64_t b, uint32_t key_bytes, cudaStream_t st) {
    PermutePlan fx;
    int rc = make_plan(layout, n, b, key_bytes, fx, ORDER_NEVER);
    if (rc) return -rc;
    if (is_veb_layout(layout) || !order_wanted(fx, ORDER_ALWAYS)) return -TL_ERROR_UNSUPPORTED;
    OrderVectors h, g;
    btree_compute_order(fx.bs, h);
    if (!btree_compute_order_device(fx.bs, st, g)) return -TL_ERROR_CUDA;
    auto eq2 = [](const std::vector<uint2> &x, const std::vector<uint2> &y) {
        if (x.size() != y.size()) return false;
        for (size_t i = 0; i < x.size(); ++i)
            if (x[i].x != y[i].x || x[i].y != y[i].y) return false;
        return true;
    };
    auto eq4 = [](const std::vector<uint4> &x, const std::vector<uint4> &y) {
        if (x.size() != y.size()) return false;
        for (size_t i = 0; i < x.size(); ++i)
            if (x[i].x != y[i].x || x[i].y != y[i].y || x[i].z != y[i].z || x[i].w != y[i].w) return false;
        return true;
    };
    bool same = eq2(h.tab, g.tab) && h.order == g.order && eq4(h.ranges, g.ranges) &&
                h.scratch_tiles == g.scratch_tiles && h.segs.size() == g.segs.size();
    for (size_t i = 0; same && i < h.segs.size(); ++i)
        same = h.segs[i].dst_len == g.segs[i].dst_len && h.segs[i].src == g.segs[i].src;
    return same ? 1 : 0;
}

// Host replay of the stream + scatter passes on a host array, one tile at a time
// in ticket order, using the same index helpers as the kernels.  Besides the
// result it counts protocol violations: a tile reading a position that was
// already overwritten, a store outside the tile's own source that is not covered
// by the tiles it waits for, a wait on a tile with a later ticket, and a final
// position or scratch slot written other than exactly once.  Test hook only.
static int emulate_permute_kb(int layout, uint64_t n, uint64_t b, uint32_t key_bytes, uint64_t *A,
                              uint64_t *violations, int order_mode) {
    PermutePlan pl;
    int rc = make_plan(layout, n, b, key_bytes, pl, ORDER_NEVER);
    if (rc) return rc;
    OrderVectors ov;  // computed here, not taken from the library's cache
    if (order_mode != ORDER_NEVER && !is_veb_layout(layout)) {
        btree_compute_order(pl.bs, ov);
        const OrderTables ot = ov.tables();
        rc = make_plan(layout, n, b, key_bytes, pl, order_mode, &ot);
        if (rc) return rc;
    }
    // tile kk's ticket precedes (or is) tile k's
    auto earlier = [&](uint64_t kk, uint64_t k) {
        if (pl.ordered) return btree_o_rank(pl.bs, kk) <= btree_o_rank(pl.bs, k);
        return pl.bs.plan == PLAN_R ? kk >= k : kk <= k;
    };
    uint64_t viol = 0;
    if (n > 1) {
        std::vector<uint64_t> scr(pl.scratch_keys, 0), tile(pl.tile_keys + 1);
        std::vector<uint8_t> readk(pl.ntiles, 0), written(n, 0);
        std::vector<uint32_t> slot_writes(pl.scratch_keys, 0), pos_writes(n, 0);
        const bool mv = is_veb_layout(pl.layout);
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
                    if (pl.ordered && !btree_o_direct(pl.bs, k, kk)) continue;  // not waited for
                    const bool ok = mv ? kk > k : pl.ordered ? earlier(kk, k) : pl.bs.plan == PLAN_R ? kk > k : kk < k;
                    if (!ok || !readk[kk]) ++viol;
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
                const BtreeStream &S = pl.bs;
                const Regime RG = btree_stream_regime(S, p0, p1);
                const uint32_t cnt = (uint32_t)(p1 - p0);
                // the runs in slot order, as warp 0 computes them, and the wait list
                TopGroup G0{}, G1{};
                const int ng = btree_stream_groups(S, p0, p1, G0, G1);
                const uint32_t nr = (uint32_t)ng * kMaxTopLevels;
                TopRun runs[kMaxTopRuns];
                uint32_t cum[kMaxTopRuns + 1], wlo[kMaxTopRuns + 1], whi[kMaxTopRuns + 1], nw = 0;
                cum[0] = 0;
                for (uint32_t sl = 0; sl < nr; ++sl) {
                    runs[sl] = btree_group_run(S, sl < kMaxTopLevels ? G0 : G1, sl % kMaxTopLevels, k);
                    cum[sl + 1] = cum[sl] + runs[sl].cnt;
                }
                uint64_t a, bq;
                std::vector<uint64_t> wl;  // plan O: the tiles the bulk stores wait for
                if (btree_tile_wait(S, p0, p1, a, bq)) {
                    if (pl.ordered) {
                        for (uint64_t kk = a; kk <= bq; ++kk) {
                            if (btree_o_direct(S, k, kk)) wl.push_back(kk);
                        }
                    } else {
                        wlo[nw] = (uint32_t)a;
                        whi[nw++] = (uint32_t)bq;
                    }
                }
                for (uint32_t sl = 0; sl < nr; ++sl)
                    if (runs[sl].cnt && btree_run_wait(S, runs[sl], a, bq)) {
                        wlo[nw] = (uint32_t)a;
                        whi[nw++] = (uint32_t)bq;
                    }
                for (uint32_t w = 0; w < nw; ++w)
                    for (uint64_t kk = wlo[w]; kk <= whi[w]; ++kk)
                        if (!earlier(kk, k) || !readk[kk]) ++viol;
                for (uint64_t kk : wl)
                    if (!earlier(kk, k) || !readk[kk]) ++viol;
                auto covered_tile = [&](uint64_t kd) {
                    if (kd == k) return true;
                    for (uint32_t w = 0; w < nw; ++w)
                        if (kd >= wlo[w] && kd <= whi[w]) return true;
                    for (uint64_t kk : wl)
                        if (kd == kk) return true;
                    return false;
                };
                auto WD = [&](uint64_t d, uint64_t v) {  // direct store, checked against the wait list
                    if (d >= n) { ++viol; return; }
                    if (!covered_tile(tile_of(d))) ++viol;
                    if (!readk[tile_of(d)]) ++viol;
                    A[d] = v;
                    written[d] = 1;
                    ++pos_writes[d];
                };
                std::vector<uint8_t> covered(cnt, 0);
                for (uint32_t o = 0; o < cnt; ++o) {
                    const uint64_t x = p0 + o;
                    uint64_t idx, ref;
                    if (RG.kind == 0) {
                        if (btree_is_top(S, x)) continue;
                        if (btree_place(S, x, idx)) WD(idx, tile[o]); else SC(idx, tile[o]);
                    } else {
                        if (RG.kind == 2 || !btree_regime_bulk(S, RG, o, idx)) continue;
                        const bool hi = RG.kind == 3 && idx >= RG.dsplit;
                        const bool to_A = hi ? RG.hi_A : RG.to_A;
                        if (RG.kind == 3 && !to_A) idx += (uint64_t)(hi ? RG.shi : RG.slo);
                        const bool direct = btree_place(S, x, ref);  // fast path == reference form
                        if (direct != to_A || ref != idx) ++viol;
                        if (to_A) WD(idx, tile[o]); else SC(idx, tile[o]);
                    }
                    covered[o] = 1;
                }
                if (cum[nr] > cnt) ++viol;
                for (uint32_t r = 0; r < nr; ++r) {
                    if (cum[r + 1] - cum[r] != runs[r].cnt) ++viol;
                    for (uint32_t e = 0; e < runs[r].cnt; ++e) {
                        const uint64_t off = btree_top_item_off(S, runs[r], e);
                        if (off >= cnt || covered[off]) { ++viol; continue; }
                        const uint64_t p = runs[r].dest0 + e;
                        const bool kdirect = btree_run_direct(S, runs[r], e);
                        const uint64_t kidx =  // the kernel's store index
                            kdirect || !pl.ordered ? p : p + (uint64_t)(e < runs[r].nlo ? runs[r].slo : runs[r].shi);
                        uint64_t ref;
                        const bool direct = btree_place(S, p0 + off, ref);
                        if (direct != kdirect || ref != kidx) ++viol;
                        if (direct) WD(kidx, tile[off]); else SC(kidx, tile[off]);
                        covered[off] = 1;
                    }
                }
                for (uint32_t o = 0; o < cnt; ++o)
                    if (!covered[o]) ++viol;
            } else {
                const MvebRegion &R = P.reg[ri];
                if (R.U == 0) {
                    for (uint64_t x = p0; x < p1; ++x) SC(R.slot_base + (x - R.src), tile[x - p0]);
                } else {
                    const unsigned char *inv = pl.mp.inv + unit_table_off(R.U);
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
            if (pl.ordered) {  // the bulk ranges and the fix pass; every slot they read written once
                std::vector<uint8_t> read_slot(pl.bs.nscratch, 0);
                for (uint64_t i = 0; i < pl.ot.nranges; ++i) {
                    const uint64_t u0 = pl.ot.ranges[i].x;
                    const uint64_t d0 = u0 * pl.tile_keys, d1 = std::min<uint64_t>(pl.ot.ranges[i].y * pl.tile_keys, n);
                    for (uint64_t d = d0; d < d1; ++d) {
                        const uint64_t sl = d + (uint64_t)btree_o_soff(pl.bs, d / pl.tile_keys);
                        if (sl >= pl.bs.nscratch || slot_writes[sl] != 1 || read_slot[sl]) { ++viol; continue; }
                        A[d] = scr[sl];
                        ++pos_writes[d];
                        read_slot[sl] = 1;
                    }
                }
                for (uint64_t i = 0; i < pl.ot.nsegs; ++i) {
                    const uint64_t d0 = pl.ot.segs[i].dst_len & kSegDstMask, len = pl.ot.segs[i].dst_len >> 48;
                    for (uint64_t e = 0; e < len; ++e) {
                        const uint64_t d = d0 + e, sl = pl.ot.segs[i].src + e;
                        // a copy takes the slot of its own position
                        if (d >= n || sl >= pl.bs.nscratch || slot_writes[sl] != 1 || read_slot[sl] ||
                            sl != d + (uint64_t)btree_o_soff(pl.bs, d / pl.tile_keys)) {
                            ++viol;
                            continue;
                        }
                        A[d] = scr[sl];
                        ++pos_writes[d];
                        read_slot[sl] = 1;
                    }
                }
                for (uint64_t c = 0; c < pl.bs.nscratch; ++c)
                    if (slot_writes[c] != read_slot[c]) ++viol;
            } else {
                for (uint64_t c = 0; c < pl.bs.nscratch; ++c)
                    if (slot_writes[c] != (btree_slot_used(pl.bs, c) ? 1u : 0u)) ++viol;
            }
            for (int j = 0; j < btree_copy_range_count(pl.bs); ++j) {
                CopyRange cr;
                if (!btree_copy_range(pl.bs, j, cr)) continue;
                for (uint64_t e = 0; e < cr.len; ++e) {
                    const uint64_t d = cr.dst + e, s1 = cr.src + e;
                    if (d >= n || s1 >= pl.bs.nscratch || !btree_slot_used(pl.bs, s1)) { ++viol; continue; }
                    A[d] = scr[s1];
                    ++pos_writes[d];
                }
            }
        } else {
            for (uint64_t s2 = 0; s2 < P.total_slots; ++s2) {
                const uint64_t rank = mveb_slot_rank(P, s2);
                if (rank == ~0ull) { if (slot_writes[s2]) ++viol; continue; }
                if (slot_writes[s2] != 1) ++viol;
                const uint64_t d = veb_pos(n, rank, P.modified != 0);
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

// Replays the ordered schedule (plan O wherever it applies) at both key widths
// (their tile sizes and scratch alignment differ) and the fixed-direction
// schedule; the results must agree.
int emulate_permute(int layout, uint64_t n, uint64_t b, uint64_t *A, uint64_t *violations) {
    std::vector<uint64_t> A4(A, A + n), Af(A, A + n);
    uint64_t v8 = 0, v4 = 0, vf = 0;
    int rc = emulate_permute_kb(layout, n, b, 8, A, &v8, ORDER_ALWAYS);
    if (!rc) rc = emulate_permute_kb(layout, n, b, 4, A4.data(), &v4, ORDER_ALWAYS);
    if (!rc) rc = emulate_permute_kb(layout, n, b, 8, Af.data(), &vf, ORDER_NEVER);
    if (rc) return rc;
    uint64_t diff = 0;
    for (uint64_t x = 0; x < n; ++x) diff += (A[x] != A4[x]) + (A[x] != Af[x]);
    if (violations) *violations = v8 + v4 + vf + diff;
    return TL_SUCCESS;
}

}  // namespace tl
