// Batched mode (no counterpart in the reference): many independent sorted
// arrays of uneven sizes, concatenated and described by an int64 offset table,
// are each permuted into a B-tree layout by ONE persistent kernel launch, and
// queried by one batch of (key, instance) pairs.
//
// Plan (built once per offset table): a setup kernel computes every instance's
// geometry and schedule (the same host/device helpers as the single-array
// path), its tile count, scratch size and copy-chunk count, and exclusive
// prefix sums of them; the host puts the instances of 64 tiles or more on the
// single-array path's ordered-tile schedule and interleaves the instances'
// tiles; a second kernel writes the owner instance of every copy chunk.
// Execute: a memset of the control words and one persistent kernel; tickets
// 0..T-1 are stream tiles (each instance's in its own schedule's order, the
// instances interleaved), tickets T.. are copy chunks (scratch -> final
// positions).  A chunk of instance j starts once all of j's tiles have stored
// (a per-instance counter, bounded wait); stream tiles never wait on chunks, so
// every wait ends.  Per size class (floor(log2 n_j)) the tile size comes from a
// tuning table that tl_batch_autotune fills by measurement.
#include <algorithm>
#include <atomic>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "batched.h"
#include "btree_order.h"
#include "btree_plan.cuh"
#include "internal.h"

namespace tl {

constexpr int kBatchThreads = 256;     // query kernel
// Permute kernel: 256 or 512 threads (tuned), compiled for 4 blocks of 256
// threads per SM (64 registers a thread).  Its plan sits in shared memory, not
// in the constant bank as the single-array kernel's does, so at the 6 blocks
// that shared memory would allow (40 registers) it spills and runs 1.3x slower
// (measured on B200: 12.6 ms against 9.4 for 2.06e9 keys).
constexpr int kBatchBlocksPerSM256 = 4;
constexpr int kBatchBlocksPerSM512 = 2;
constexpr int kMaxClass = 48;

struct alignas(16) BatchInst {
    BtreeStream S;
    uint64_t off;          // first key of the instance
    uint64_t tile_base;    // first of the instance's tile flags
    uint64_t scr_base;     // first scratch slot (same 16-byte offset as the instance's keys)
    uint64_t chunk_base;   // first global copy chunk
    uint64_t nchunks;
    uint64_t item_base;    // ordered schedule: the instance's copy items in the plan's item list
    uint64_t nitems;
};

// Ordered-schedule instances (from kBatchOrderMinTiles tiles, as the single-array
// permutation): their scratch keys go back as copy items, a warp each (whole-tile
// runs in pieces of kRangePiece keys, and the fix pass's segments), grouped into
// copy chunks of at most kCopyChunk keys and kChunkItemsMax items.
constexpr uint64_t kBatchOrderMinTiles = 64;
constexpr uint64_t kChunkItemsMax = 64;
constexpr uint64_t kRangePiece = 2048;
// An instance takes the ordered schedule only if that moves at most this share
// of the scratch keys of its fixed-direction schedule: in the batched kernel
// (plan in shared memory, 64 registers) an ordered tile costs more instructions
// than a fixed one, and fewer bytes pay for them only where they are many fewer.
// Measured on B200, 4096 arrays of 2^10..2^22 keys: b = 16 9.02 ms at 0.3
// against 9.51 fixed and 9.39 ordered everywhere; b = 8 9.34 / 9.42 / 9.69;
// b = 1 11.76 / 11.76 / 12.37.
constexpr double kOrderGain = 0.3;
constexpr uint64_t kInterleaveRun = 1;  // stream tiles an instance takes in a row
static_assert(sizeof(BatchInst) % 16 == 0, "BatchInst is copied to shared memory in 16-byte words");

struct BatchTotals {
    uint64_t tiles, chunks, scratch, max_tile;
};

struct tl_batch_plan_impl {
    uint32_t num = 0, key_bytes = 8;
    uint64_t b = 8;
    BatchInst *inst = nullptr;   // device
    BatchTotals tot{};
    uint32_t tile_keys[kMaxClass];
    uint32_t pin_levels[kMaxClass];  // query: top levels pinned in shared memory per size class
    uint32_t query_chunk = 2048;     // queries per CTA work item
    uint32_t threads = 256;          // permute kernel block size
    uint32_t *owner = nullptr;   // device: owner instance of every tile ticket, then of every copy chunk
    uint32_t *tile = nullptr;    // device: the tile of its owner every tile ticket processes
    char *otab = nullptr;        // device: the ordered instances' tile tables (uint2 tab, then uint32 order)
    FixSeg *items = nullptr;     // device: the ordered instances' copy items
    uint64_t *citem = nullptr;   // device: first copy item of every copy chunk of an ordered instance
    uint64_t ordered = 0;        // instances on the ordered schedule
    uint64_t ordered_keys = 0;   // their keys
    uint64_t off_flags = 0, off_done = 0, off_ctrl = 0, ws_bytes = 0;
    uint64_t total_keys = 0;
};

// ---------------------------------------------------------------- setup
__global__ void __launch_bounds__(256) batch_setup_kernel(const int64_t *__restrict__ offsets, uint32_t num, uint64_t b,
                                                          uint32_t key_bytes, FastDiv64 fd, FastDiv32 fd32,
                                                          FastDiv32 fd32b, const __grid_constant__ PowDivs pdivs,
                                                          const uint32_t *__restrict__ tile_keys,
                                                          BatchInst *__restrict__ inst, BatchTotals *__restrict__ tot) {
    // one block: per-instance plans, then exclusive scans in instance order
    __shared__ unsigned long long s_part[3][1024];
    const uint32_t T = blockDim.x;
    const uint32_t per = (num + T - 1) / T;
    const uint32_t j0 = threadIdx.x * per, j1 = min(num, j0 + per);
    const uint64_t vec = 16 / key_bytes;
    unsigned long long st = 0, ss = 0, sc = 0;
    for (uint32_t j = j0; j < j1; ++j) {
        BatchInst I;
        memset(&I, 0, sizeof I);
        const uint64_t n = (uint64_t)(offsets[j + 1] - offsets[j]);
        I.off = (uint64_t)offsets[j];
        I.S.g = make_btree_geom(n, b);
        I.S.fd = fd;
        I.S.fd32 = fd32;
        I.S.fd32b = fd32b;
        btree_set_pow_divs(I.S, pdivs);
        const uint32_t cls = n ? bit_length(n) - 1 : 0;
        I.S.tile_keys = tile_keys[cls < kMaxClass ? cls : kMaxClass - 1];  // a power of two
        I.S.tile_shift = (uint32_t)__ffsll((long long)I.S.tile_keys) - 1;
        I.S.ntiles = (n + I.S.tile_keys - 1) / I.S.tile_keys;
        btree_choose_plan(I.S, key_bytes);
        if (n <= 1) {
            I.S.ntiles = 0;
            I.S.nscratch = 0;
        }
        uint64_t ncopy = 0;
        for (int k = 0; k < btree_copy_range_count(I.S); ++k) {
            CopyRange r;
            if (btree_copy_range(I.S, k, r)) ncopy += r.len;
        }
        I.nchunks = I.S.nscratch ? (ncopy + kCopyChunk - 1) / kCopyChunk : 0;
        st += I.S.ntiles;
        ss += I.S.nscratch ? I.S.nscratch + vec - 1 : 0;  // room to align the base
        sc += I.nchunks;
        inst[j] = I;
    }
    s_part[0][threadIdx.x] = st;
    s_part[1][threadIdx.x] = ss;
    s_part[2][threadIdx.x] = sc;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long a = 0, c = 0, d = 0;
        for (uint32_t t = 0; t < T; ++t) {
            const unsigned long long x = s_part[0][t], y = s_part[1][t], z = s_part[2][t];
            s_part[0][t] = a;
            s_part[1][t] = c;
            s_part[2][t] = d;
            a += x;
            c += y;
            d += z;
        }
        tot->tiles = a;
        tot->scratch = c;
        tot->chunks = d;
        uint64_t mt = 0;
        for (int k = 0; k < kMaxClass; ++k) mt = max(mt, (uint64_t)tile_keys[k]);
        tot->max_tile = mt;
    }
    __syncthreads();
    unsigned long long bt = s_part[0][threadIdx.x], bs = s_part[1][threadIdx.x], bc = s_part[2][threadIdx.x];
    for (uint32_t j = j0; j < j1; ++j) {
        const uint64_t ns = inst[j].S.nscratch;
        inst[j].tile_base = bt;
        inst[j].scr_base = bs + ((inst[j].off % vec) + vec - (bs % vec)) % vec;
        inst[j].chunk_base = bc;
        bt += inst[j].S.ntiles;
        bs += ns ? ns + vec - 1 : 0;
        bc += inst[j].nchunks;
    }
}

// owner[tiles + c] = instance of copy chunk c; tile[t], for a tile ticket t, from
// the owner's own ticket (as the host interleaved them) to the tile it names
// under the owner's schedule.  (The owners of tile tickets come from the host.)
__global__ void batch_owner_kernel(const BatchInst *__restrict__ inst, uint32_t num, uint64_t tiles,
                                   uint32_t *__restrict__ owner, uint32_t *__restrict__ tile) {
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t i0 = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x, ni = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t t = i0; t < tiles; t += ni) tile[t] = (uint32_t)btree_tile_of_ticket(inst[owner[t]].S, tile[t]);
    for (uint64_t j = i0 >> 5; j < num; j += ni >> 5) {
        const BatchInst &I = inst[j];
        for (uint64_t c = lane; c < I.nchunks; c += 32) owner[tiles + I.chunk_base + c] = (uint32_t)j;
    }
}

// ---------------------------------------------------------------- permute
// Ordered schedule: copy chunk c of instance I is a run of its copy items, a warp each.
template <typename K>
static __device__ __forceinline__ void batch_copy_items(K *__restrict__ keys, K *__restrict__ scr, const BatchInst &I,
                                                     const FixSeg *__restrict__ items,
                                                     const uint64_t *__restrict__ citem, uint64_t c) {
    const uint64_t i0 = citem[I.chunk_base + c];
    const uint64_t i1 = c + 1 < I.nchunks ? citem[I.chunk_base + c + 1] : I.item_base + I.nitems;
    K *const dst = keys + I.off;
    const K *const src = scr + I.scr_base;
    for (uint64_t i = i0 + (threadIdx.x >> 5); i < i1; i += blockDim.x >> 5) {
        const uint64_t dl = __ldg(reinterpret_cast<const unsigned long long *>(&items[i].dst_len));
        const uint64_t so = __ldg(reinterpret_cast<const unsigned long long *>(&items[i].src));
        warp_copy_keys(dst + (dl & kSegDstMask), src + so, 0, (uint32_t)(dl >> 48));
    }
}

// Fixed directions: copy chunk c of instance I is kCopyChunk keys of its copy
// ranges, taken as one concatenated range.
template <typename K>
static __device__ __forceinline__ void batch_copy_ranges(K *__restrict__ keys, K *__restrict__ scr, const BatchInst &I,
                                                      uint64_t c) {
    const uint64_t lo = c * kCopyChunk, hi = lo + kCopyChunk;
    uint64_t acc = 0;
    const int nr = btree_copy_range_count(I.S);
    for (int q = 0; q < nr && acc < hi; ++q) {
        CopyRange r;
        if (!btree_copy_range(I.S, q, r)) continue;
        const uint64_t a = lo > acc ? lo - acc : 0;
        const uint64_t e = min(hi - acc, r.len);
        if (a < e) copy_keys(keys + I.off + r.dst + a, scr + I.scr_base + r.src + a, e - a, 0, 1);
        acc += r.len;
    }
}

constexpr uint32_t kNoInst = 0xFFFFFFFFu;
constexpr uint32_t kPlanWords = sizeof(BatchInst) / 16;

// Warps 1.. copy instance j's plan to a shared-memory buffer with cp.async (they
// wait for it with their tile's copies, or explicitly after a copy chunk).
__device__ __forceinline__ void prefetch_plan(const BatchInst *inst, uint32_t j, unsigned char *buf) {
    if (threadIdx.x < 32) return;
    const char *src = reinterpret_cast<const char *>(inst + j);
    const uint32_t dst = (uint32_t)__cvta_generic_to_shared(buf);
    for (uint32_t w = threadIdx.x - 32; w < kPlanWords; w += blockDim.x - 32)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst + w * 16), "l"(src + (size_t)w * 16)
                     : "memory");
    asm volatile("cp.async.commit_group;" ::: "memory");
}

// Work items in ticket order; a block holds four tickets: the item it works
// on, the next (its owner and tile known, its owner's plan copied to the
// second plan buffer while the current item runs), the one after (its owner
// copied to shared memory while the current item runs) and a fourth (the
// atomic claiming it in flight).  Thread 0 starts those copies (cp.async, no
// registers held across the item) as an item starts; between two items it
// alone releases the finished tile to its instance's copy chunks (fence, then
// the done counter) and moves the pipeline on, one barrier on either side.
// Holding tickets ahead cannot stall the launch: the smallest ticket held and
// not yet done is always some block's current item, and an item waits only
// for smaller tickets.
template <typename K, int kThreads, int kMinBlocks>
__global__ void __launch_bounds__(kThreads, kMinBlocks)
batch_permute_kernel(K *__restrict__ keys, K *__restrict__ scr, const BatchInst *__restrict__ inst,
                     const uint32_t *__restrict__ owner, const uint32_t *__restrict__ tile,
                     const FixSeg *__restrict__ items, const uint64_t *__restrict__ citem, BatchTotals tot,
                     Ctrl *ctrl, WaitCfg wc, unsigned int *flags, unsigned int *done) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    K *sm = tile_smem<K>(smem_raw);
    __shared__ __align__(16) unsigned char s_plan[2][sizeof(BatchInst)];
    __shared__ unsigned long long s_t;  // the current ticket
    __shared__ uint32_t s_j, s_k;       // its owner and (a tile) its tile
    __shared__ uint32_t s_nj;           // the owner of the next ticket (kNoInst past the end)
    __shared__ uint32_t s_held[2];      // the instance whose plan each buffer holds
    __shared__ uint32_t s_k1, s_j2;     // the tile of the next ticket, the owner of the one after
    __shared__ int s_ok;
    __shared__ TileShared ts;
    const uint64_t total = tot.tiles + tot.chunks;
    uint32_t t1 = 0, t2 = 0;  // thread 0: the next ticket and the one after (below 2^31, as built)
    if (threadIdx.x == 0) {
        const unsigned long long t0 = atomicAdd(&ctrl->ticket, 1ull);
        t1 = (uint32_t)atomicAdd(&ctrl->ticket, 1ull);
        t2 = (uint32_t)atomicAdd(&ctrl->ticket, 1ull);
        s_t = t0;
        s_j = t0 < total ? owner[t0] : kNoInst;
        s_k = t0 < tot.tiles ? tile[t0] : 0;
        s_nj = t1 < total ? owner[t1] : kNoInst;
        s_held[0] = s_held[1] = kNoInst;
    }
    __syncthreads();
    while (s_t < total) {
        const unsigned long long t = s_t;
        const uint32_t j = s_j, nj = s_nj;
        uint32_t t3 = 0;
        if (threadIdx.x == 0) {  // read as the item ends
            if (t1 < tot.tiles)
                asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"((uint32_t)__cvta_generic_to_shared(&s_k1)),
                             "l"(tile + t1) : "memory");
            if (t2 < total)
                asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"((uint32_t)__cvta_generic_to_shared(&s_j2)),
                             "l"(owner + t2) : "memory");
            asm volatile("cp.async.commit_group;" ::: "memory");
            t3 = (uint32_t)atomicAdd(&ctrl->ticket, 1ull);
        }
        int cb = s_held[0] == j ? 0 : s_held[1] == j ? 1 : -1;
        if (cb < 0) {  // not prefetched (the block's first item): copy it now
            cb = s_held[0] == nj ? 1 : 0;
            const uint4 *src = reinterpret_cast<const uint4 *>(inst + j);
            uint4 *dst = reinterpret_cast<uint4 *>(s_plan[cb]);
            for (uint32_t w = threadIdx.x; w < kPlanWords; w += blockDim.x) dst[w] = src[w];
            __syncthreads();
            if (threadIdx.x == 0) s_held[cb] = j;  // read again only after the next barrier
        }
        const BatchInst &I = *reinterpret_cast<const BatchInst *>(s_plan[cb]);
        const bool pf = nj != kNoInst && nj != j && s_held[1 - cb] != nj;
        if (pf) prefetch_plan(inst, nj, s_plan[1 - cb]);
        const bool is_tile = t < tot.tiles;
        if (is_tile) {
            btree_stream_tile(I.S, keys + I.off, scr + I.scr_base, flags + I.tile_base, ctrl, wc, s_k, sm, ts);
        } else {
            if (threadIdx.x == 0) s_ok = wait_flag(&done[j], (unsigned int)I.S.ntiles, ctrl, wc) ? 1 : 0;
            __syncthreads();
            if (s_ok) {
                const uint64_t c = t - tot.tiles - I.chunk_base;
                if (I.S.plan == PLAN_O)
                    batch_copy_items(keys, scr, I, items, citem, c);
                else
                    batch_copy_ranges(keys, scr, I, c);
            }
            load_tile_wait();  // the plan prefetch, where there is one
        }
        __syncthreads();  // the item is done (every store of a tile issued); a prefetched plan has landed
        if (threadIdx.x == 0) {
            const unsigned long long n = t1;
            load_tile_wait();
            const uint32_t k1 = t1 < tot.tiles ? s_k1 : 0, j2 = t2 < total ? s_j2 : kNoInst;
            if (is_tile) {  // the tile's stores, every thread's, before its count
                __threadfence();
                atomicAdd(&done[j], 1u);
            }
            if (pf) s_held[1 - cb] = nj;
            s_t = n;
            s_j = nj;
            s_k = k1;
            s_nj = j2;
            t1 = t2;
            t2 = t3;
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------- queries
// Queries are grouped by instance (counting sort: histogram, scan, scatter) so
// that a CTA's work item mostly belongs to one instance; the CTA then pins that
// instance's top levels in shared memory (depth from the size-class table).
__global__ void batch_hist_kernel(const uint32_t *__restrict__ qinst, uint64_t q, uint32_t num,
                                  unsigned int *__restrict__ count) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < q; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t j = qinst[i];
        if (j < num) atomicAdd(&count[j], 1u);
    }
}

__global__ void batch_scan_kernel(const unsigned int *__restrict__ count, uint32_t num,
                                  unsigned long long *__restrict__ start) {
    __shared__ unsigned long long s_part[1024];
    const uint32_t T = blockDim.x, per = (num + T - 1) / T;
    const uint32_t j0 = threadIdx.x * per, j1 = min(num, j0 + per);
    unsigned long long acc = 0;
    for (uint32_t j = j0; j < j1; ++j) acc += count[j];
    s_part[threadIdx.x] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long a = 0;
        for (uint32_t t = 0; t < T; ++t) {
            const unsigned long long x = s_part[t];
            s_part[t] = a;
            a += x;
        }
        start[num] = a;
    }
    __syncthreads();
    unsigned long long p = s_part[threadIdx.x];
    for (uint32_t j = j0; j < j1; ++j) {
        start[j] = p;
        p += count[j];
    }
}

template <typename K>
__global__ void batch_bucket_kernel(const K *__restrict__ Q, const uint32_t *__restrict__ qinst, uint64_t q,
                                    uint32_t num, unsigned long long *__restrict__ cursor, K *__restrict__ sq,
                                    uint32_t *__restrict__ sinst, uint64_t *__restrict__ sidx) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < q; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t j = qinst[i];
        if (j >= num) continue;
        const unsigned long long p = atomicAdd(&cursor[j], 1ull);
        sq[p] = Q[i];
        sinst[p] = j;
        sidx[p] = i;
    }
}

template <typename K>
__global__ void __launch_bounds__(kBatchThreads)
batch_query_kernel(const K *__restrict__ keys, const BatchInst *__restrict__ inst, const K *__restrict__ sq,
                   const uint32_t *__restrict__ sinst, const uint64_t *__restrict__ sidx,
                   const unsigned long long *__restrict__ nvalid, uint32_t chunk,
                   const uint32_t *__restrict__ pin_levels, uint32_t pin_cap, uint64_t *__restrict__ ans) {
    const uint64_t q = *nvalid;  // queries with a valid instance id (sorted first)
    extern __shared__ __align__(16) unsigned char smem_raw[];
    K *sm = reinterpret_cast<K *>(smem_raw);
    __shared__ uint32_t s_j, s_one;
    __shared__ uint64_t s_P;
    const uint64_t nchunks = (q + chunk - 1) / chunk;
    for (uint64_t ck = blockIdx.x; ck < nchunks; ck += gridDim.x) {
        const uint64_t q0 = ck * chunk, q1 = min(q, q0 + chunk);
        __syncthreads();
        if (threadIdx.x == 0) {
            s_j = sinst[q0];
            s_one = sinst[q1 - 1] == s_j;
            uint64_t P = 0;
            if (s_one) {
                const BtreeStream &S = inst[s_j].S;
                const uint32_t cls = S.g.n ? bit_length(S.g.n) - 1 : 0;
                const uint32_t L = pin_levels[cls < kMaxClass ? cls : kMaxClass - 1];
                const uint32_t LL = L < S.g.h + 1 ? L : S.g.h + 1;
                P = L ? min(S.g.n, S.g.pw[LL] - 1) : 0;
                if (P > pin_cap) P = 0;
            }
            s_P = P;
        }
        __syncthreads();
        const uint64_t P = s_P;
        if (P) {
            const K *A = keys + inst[s_j].off;
            for (uint64_t x = threadIdx.x; x < P; x += blockDim.x) sm[x] = __ldg(A + x);
            __syncthreads();
        }
        for (uint64_t i = q0 + threadIdx.x; i < q1; i += blockDim.x) {
            const uint32_t j = sinst[i];
            const BtreeStream &S = inst[j].S;
            const K *A = keys + inst[j].off;
            const uint64_t n = S.g.n, b = S.g.b;
            const uint64_t PP = (s_one && j == s_j) ? P : 0;
            const K qv = sq[i];
            uint64_t node = 0, res = n;
            const uint64_t cmax = (n + 1) / (b + 1);
            // node rows in 32-byte (or 16-byte) loads where the instance's keys
            // and its nodes start on such a boundary, else key by key
            const uintptr_t abase = reinterpret_cast<uintptr_t>(A);
            const uint32_t vb = (abase & 31) == 0 && (b * sizeof(K)) % 32 == 0   ? 32u
                                : (abase & 15) == 0 && (b * sizeof(K)) % 16 == 0 ? 16u
                                                                                  : 0u;
            while (node < n) {
                const uint64_t valid = min(b, n - node);
                uint32_t lt = 0;
                bool eq = false;
                if (vb && valid == b && node >= PP) {
                    const uint32_t kpl = vb / sizeof(K), nl = (uint32_t)(b / kpl);
#pragma unroll 4
                    for (uint32_t j = 0; j < nl; ++j) {
                        K v[32 / sizeof(K)];
                        if (vb == 32) {
                            ldg32(A + node + (uint64_t)j * kpl, v);
                        } else {
                            const uint4 x = __ldg(reinterpret_cast<const uint4 *>(A + node + (uint64_t)j * kpl));
                            const K *kx = reinterpret_cast<const K *>(&x);
#pragma unroll
                            for (int e = 0; e < (int)(16 / sizeof(K)); ++e) v[e] = kx[e];
                        }
#pragma unroll
                        for (int e = 0; e < (int)(32 / sizeof(K)); ++e)
                            if (vb == 32 || e < (int)(16 / sizeof(K))) {
                                lt += v[e] < qv;
                                eq |= v[e] == qv;
                            }
                    }
                } else {
                    for (uint64_t s = 0; s < valid; ++s) {
                        const uint64_t p = node + s;
                        const K cur = p < PP ? sm[p] : __ldg(A + p);
                        lt += cur < qv;
                        eq |= cur == qv;
                    }
                }
                if (eq) {  // keys are unique: the equal key sits at slot lt
                    res = node + lt;
                    break;
                }
                if (node + 1 > cmax) break;
                node = (node + 1) * (b + 1) + (uint64_t)lt * b - 1;
            }
            ans[sidx[i]] = res;
        }
    }
}

// ---------------------------------------------------------------- host
static int batch_sms() {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return sms;
}

static void default_tuning(tl_batch_plan_impl &P) {
    for (int c = 0; c < kMaxClass; ++c) {
        P.tile_keys[c] = (uint32_t)(32768 / P.key_bytes);
        P.pin_levels[c] = 3;
    }
    P.query_chunk = 2048;
}

static void free_order_buffers(tl_batch_plan_impl &P) {
    if (P.otab) cudaFree(P.otab);
    if (P.items) cudaFree(P.items);
    if (P.citem) cudaFree(P.citem);
    P.otab = nullptr;
    P.items = nullptr;
    P.citem = nullptr;
    P.ordered = P.ordered_keys = 0;
}

// A device copy of v, landed when this returns (copied on st, then waited for:
// a plain cudaMemcpy from pageable memory may return before its DMA lands).
template <typename T>
static int upload(T *&dst, const std::vector<T> &v, cudaStream_t st) {
    if (cudaMalloc(reinterpret_cast<void **>(&dst), std::max<size_t>(v.size(), 1) * sizeof(T)) != cudaSuccess) {
        cudaGetLastError();
        dst = nullptr;
        return TL_ERROR_OUT_OF_MEMORY;
    }
    if (!v.empty()) TL_CUDA_TRY(cudaMemcpyAsync(dst, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, st));
    TL_CUDA_TRY(cudaStreamSynchronize(st));
    return TL_SUCCESS;
}

// Keys through scratch under an instance's fixed-direction schedule and under
// the ordered one.
static uint64_t fixed_scratch_keys(const BtreeStream &S) {
    uint64_t c = 0;
    CopyRange r;
    for (int k = 0; k < btree_copy_range_count(S); ++k)
        if (btree_copy_range(S, k, r)) c += r.len;
    return c;
}

static uint64_t order_scratch_keys(const BtreeStream &S, const OrderVectors &v) {
    uint64_t c = 0;
    for (const uint4 &r : v.ranges)
        c += std::min<uint64_t>((uint64_t)r.y * S.tile_keys, S.g.n) - (uint64_t)r.x * S.tile_keys;
    for (const FixSeg &f : v.segs) c += f.dst_len >> 48;
    return c;
}

// Puts every instance of kBatchOrderMinTiles tiles or more (with a top tree) on
// the ordered schedule of the single-array permutation: its tile order and
// scratch tables are computed on the host (instances shared among a few host
// threads), its scratch keys listed as copy items and grouped into chunks; then
// every instance's scratch and chunk bases are recomputed in instance order
// (the same rules as batch_setup_kernel) and the plan is written back.
static int order_instances(tl_batch_plan_impl &P, const std::vector<int64_t> &off, cudaStream_t st) {
    free_order_buffers(P);
    if (fixed_schedule_only()) return TL_SUCCESS;
    std::vector<uint32_t> cand;
    for (uint32_t j = 0; j < P.num; ++j) {
        const uint64_t n = (uint64_t)(off[j + 1] - off[j]);
        const uint32_t cls = n ? bit_length(n) - 1 : 0;
        const uint64_t tk = P.tile_keys[cls < kMaxClass ? cls : kMaxClass - 1];
        if ((n + tk - 1) / tk >= kBatchOrderMinTiles) cand.push_back(j);
    }
    if (cand.empty()) return TL_SUCCESS;
    std::vector<BatchInst> h(P.num);
    TL_CUDA_TRY(cudaMemcpyAsync(h.data(), P.inst, h.size() * sizeof(BatchInst), cudaMemcpyDeviceToHost, st));
    TL_CUDA_TRY(cudaStreamSynchronize(st));
    if (P.b >= 2)  // the host's inverse map (sorted rank of a position) divides by b
        for (uint32_t j : cand) h[j].S.fdb = FastDiv64(P.b);
    std::vector<OrderVectors> ov(cand.size());
    std::vector<int32_t> ord_of(P.num, -1);
    {
        std::atomic<size_t> next{0};
        auto work = [&] {
            for (size_t i; (i = next.fetch_add(1)) < cand.size();) {
                const BtreeStream &S = h[cand[i]].S;
                if (S.g.h < 1 || S.ntiles < kBatchOrderMinTiles || S.ntiles >= (1ull << 32)) continue;
                btree_compute_order(S, ov[i]);
                if (!ordered_schedule_forced() &&
                    order_scratch_keys(S, ov[i]) > kOrderGain * (double)fixed_scratch_keys(S))
                    ov[i] = OrderVectors();
            }
        };
        const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
        const size_t nth = std::min<size_t>({(size_t)hw, (size_t)16, cand.size()});
        std::vector<std::thread> pool;
        for (size_t k = 1; k < nth; ++k) pool.emplace_back(work);
        work();
        for (auto &t : pool) t.join();
    }
    // the tables of the ordered instances, each its tab then its order (8-byte aligned)
    std::vector<size_t> toff(cand.size(), 0);
    size_t tbytes = 0;
    for (size_t i = 0; i < cand.size(); ++i) {
        if (ov[i].order.empty()) continue;
        ord_of[cand[i]] = (int32_t)i;
        toff[i] = tbytes;
        const size_t N = ov[i].order.size();
        tbytes += N * sizeof(uint2) + (N * sizeof(uint32_t) + 7) / 8 * 8;
    }
    if (!tbytes) return TL_SUCCESS;
    std::vector<char> tb(tbytes, 0);
    for (size_t i = 0; i < cand.size(); ++i) {
        if (ord_of[cand[i]] < 0) continue;
        const size_t N = ov[i].order.size();
        memcpy(tb.data() + toff[i], ov[i].tab.data(), N * sizeof(uint2));
        memcpy(tb.data() + toff[i] + N * sizeof(uint2), ov[i].order.data(), N * sizeof(uint32_t));
    }
    int rc = upload(P.otab, tb, st);
    if (rc) return rc;
    std::vector<FixSeg> items;
    std::vector<uint64_t> citem;
    const uint64_t vec = 16 / P.key_bytes;
    uint64_t bs = 0;
    for (uint32_t j = 0; j < P.num; ++j) {
        BatchInst &I = h[j];
        I.chunk_base = citem.size();
        if (ord_of[j] >= 0) {
            const OrderVectors &v = ov[ord_of[j]];
            const size_t N = v.order.size();
            const char *t = P.otab + toff[ord_of[j]];
            btree_set_ordered(I.S, reinterpret_cast<const uint2 *>(t),
                              reinterpret_cast<const uint32_t *>(t + N * sizeof(uint2)), v.scratch_tiles);
            const uint64_t T = I.S.tile_keys, n = I.S.g.n;
            I.item_base = items.size();
            for (const uint4 &r : v.ranges)  // whole-tile runs, in pieces
                for (uint64_t d = (uint64_t)r.x * T, s = (uint64_t)r.z * T, e = std::min<uint64_t>((uint64_t)r.y * T, n);
                     d < e;) {
                    const uint64_t len = std::min<uint64_t>(kRangePiece, e - d);
                    items.push_back(FixSeg{d | (len << 48), s});
                    d += len;
                    s += len;
                }
            items.insert(items.end(), v.segs.begin(), v.segs.end());
            I.nitems = items.size() - I.item_base;
            I.nchunks = 0;
            uint64_t keys = kCopyChunk, cnt = 0;
            for (uint64_t k = I.item_base; k < items.size(); ++k) {
                const uint64_t len = items[k].dst_len >> 48;
                if (keys + len > kCopyChunk || cnt == kChunkItemsMax) {
                    citem.push_back(k);
                    ++I.nchunks;
                    keys = cnt = 0;
                }
                keys += len;
                ++cnt;
            }
            ++P.ordered;
            P.ordered_keys += n;
        } else {
            citem.resize(citem.size() + I.nchunks, 0);  // plan R / L chunks: not read
        }
        const uint64_t ns = I.S.nscratch;
        I.scr_base = bs + ((I.off % vec) + vec - (bs % vec)) % vec;
        bs += ns ? ns + vec - 1 : 0;
    }
    P.tot.scratch = bs;
    P.tot.chunks = citem.size();
    rc = upload(P.items, items, st);
    if (!rc) rc = upload(P.citem, citem, st);
    if (!rc) {
        TL_CUDA_TRY(cudaMemcpyAsync(P.inst, h.data(), h.size() * sizeof(BatchInst), cudaMemcpyHostToDevice, st));
        TL_CUDA_TRY(cudaStreamSynchronize(st));
    }
    if (rc) free_order_buffers(P);
    return rc;
}

// The order in which the persistent kernel takes the stream tiles: each
// instance's tiles in its own ticket order, the instances interleaved in
// proportion to their tile counts, kInterleaveRun tiles at a time.  A tile only
// waits for tiles of its own instance with smaller tickets; interleaved, those
// were claimed some thousands of tickets earlier and have long been read,
// where instance after instance they would be the tiles just claimed, often
// still loading (measured on B200, 4096 arrays of 2^10..2^22 keys, b = 8: the
// waits that found their flag unset fall from 4.2e5 to 1e4 and the launch from
// 11.1 to 9.6 ms).  Longer runs, which reload the owner's plan into shared
// memory less often, measured slower (runs of 4: 9.7 ms).
static int interleave_tiles(const tl_batch_plan_impl &P, const std::vector<int64_t> &off,
                            std::vector<uint32_t> &own, std::vector<uint32_t> &loc) {
    struct Run {
        double key;  // the instance's progress at the run's middle
        uint32_t j, r;
    };
    const uint64_t G = kInterleaveRun;
    std::vector<Run> runs;
    std::vector<uint64_t> nt(P.num);
    uint64_t sum = 0;
    for (uint32_t j = 0; j < P.num; ++j) {
        const uint64_t n = (uint64_t)(off[j + 1] - off[j]);
        const uint32_t cls = n ? bit_length(n) - 1 : 0;
        const uint64_t tk = P.tile_keys[cls < kMaxClass ? cls : kMaxClass - 1];
        nt[j] = n <= 1 ? 0 : (n + tk - 1) / tk;  // as batch_setup_kernel
        sum += nt[j];
        const uint64_t R = (nt[j] + G - 1) / G;
        for (uint64_t r = 0; r < R; ++r) runs.push_back(Run{((double)r + 0.5) / (double)R, j, (uint32_t)r});
    }
    // tile indices and the kernel's tickets are 32-bit
    if (sum != P.tot.tiles || sum + P.tot.chunks >= (1ull << 31)) return TL_ERROR_UNSUPPORTED;
    std::stable_sort(runs.begin(), runs.end(), [](const Run &a, const Run &b) { return a.key < b.key; });
    own.clear();
    loc.clear();
    own.reserve(sum);
    loc.reserve(sum);
    for (const Run &q : runs)
        for (uint64_t i = (uint64_t)q.r * G, e = std::min<uint64_t>(i + G, nt[q.j]); i < e; ++i) {
            own.push_back(q.j);
            loc.push_back((uint32_t)i);
        }
    return TL_SUCCESS;
}

// Frees a stream-ordered temporary on every exit path.
struct AsyncBuffer {
    void *p = nullptr;
    cudaStream_t st;
    explicit AsyncBuffer(cudaStream_t s) : st(s) {}
    ~AsyncBuffer() {
        if (p) cudaFreeAsync(p, st);
    }
};

static int build_plan(tl_batch_plan_impl &P, const int64_t *dev_offsets, cudaStream_t st) {
    AsyncBuffer tk_buf(st), tot_buf(st);
    keep_pool_memory();
    TL_CUDA_TRY(cudaMallocAsync(&tk_buf.p, sizeof(P.tile_keys), st));
    TL_CUDA_TRY(cudaMallocAsync(&tot_buf.p, sizeof(BatchTotals), st));
    uint32_t *d_tk = static_cast<uint32_t *>(tk_buf.p);
    BatchTotals *d_tot = static_cast<BatchTotals *>(tot_buf.p);
    TL_CUDA_TRY(cudaMemcpyAsync(d_tk, P.tile_keys, sizeof(P.tile_keys), cudaMemcpyHostToDevice, st));
    batch_setup_kernel<<<1, 256, 0, st>>>(dev_offsets, P.num, P.b, P.key_bytes, FastDiv64(P.b + 1),
                                           FastDiv32((uint32_t)(P.b + 1)),
                                           P.b >= 2 ? FastDiv32((uint32_t)P.b) : FastDiv32(), make_pow_divs(P.b), d_tk,
                                           P.inst, d_tot);
    TL_CUDA_TRY(cudaGetLastError());
    int64_t last = 0;
    TL_CUDA_TRY(cudaMemcpyAsync(&P.tot, d_tot, sizeof(BatchTotals), cudaMemcpyDeviceToHost, st));
    TL_CUDA_TRY(cudaMemcpyAsync(&last, dev_offsets + P.num, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    TL_CUDA_TRY(cudaStreamSynchronize(st));
    P.total_keys = (uint64_t)last;
    std::vector<int64_t> off(P.num + 1);
    TL_CUDA_TRY(cudaMemcpyAsync(off.data(), dev_offsets, off.size() * sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    TL_CUDA_TRY(cudaStreamSynchronize(st));
    int rc = order_instances(P, off, st);
    if (rc) return rc;
    std::vector<uint32_t> own, loc;
    rc = interleave_tiles(P, off, own, loc);
    if (rc) return rc;
    if (P.owner) cudaFreeAsync(P.owner, st);
    if (P.tile) cudaFreeAsync(P.tile, st);
    P.owner = P.tile = nullptr;
    const uint64_t nowner = P.tot.tiles + P.tot.chunks;
    if (nowner) {
        keep_pool_memory();
        TL_CUDA_TRY(cudaMallocAsync(reinterpret_cast<void **>(&P.owner), nowner * sizeof(uint32_t), st));
        TL_CUDA_TRY(cudaMallocAsync(reinterpret_cast<void **>(&P.tile),
                                    std::max<uint64_t>(P.tot.tiles, 1) * sizeof(uint32_t), st));
        if (P.tot.tiles) {
            TL_CUDA_TRY(cudaMemcpyAsync(P.owner, own.data(), own.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
            TL_CUDA_TRY(cudaMemcpyAsync(P.tile, loc.data(), loc.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
        }
        const uint64_t work = std::max<uint64_t>((uint64_t)P.num * 32, P.tot.tiles);
        const unsigned g = (unsigned)std::min<uint64_t>((work + 255) / 256, (uint64_t)batch_sms() * 8);
        batch_owner_kernel<<<g, 256, 0, st>>>(P.inst, P.num, P.tot.tiles, P.owner, P.tile);
        TL_CUDA_TRY(cudaGetLastError());
        TL_CUDA_TRY(cudaStreamSynchronize(st));  // the plan is complete when this returns, for any stream
    }
    auto al = [](uint64_t x) { return (x + 255) / 256 * 256; };
    // + 16 bytes: the scratch starts at the keys' own offset within 16 bytes
    P.off_flags = al(P.tot.scratch * P.key_bytes + 16);
    P.off_done = P.off_flags + al(P.tot.tiles * sizeof(unsigned int));
    P.off_ctrl = P.off_done + al((uint64_t)P.num * sizeof(unsigned int));
    P.ws_bytes = P.off_ctrl + al(sizeof(Ctrl));
    return TL_SUCCESS;
}

int batch_plan_create(const int64_t *dev_offsets, uint32_t num, uint64_t b, uint32_t key_bytes, cudaStream_t st,
                      tl_batch_plan **out) {
    if (!dev_offsets || !out || num == 0 || num > (1u << 24) || b == 0 || b >= (1u << 20) ||
        (key_bytes != 4 && key_bytes != 8))
        return TL_ERROR_INVALID_VALUE;
    auto *P = new tl_batch_plan_impl;
    P->num = num;
    P->b = b;
    P->key_bytes = key_bytes;
    default_tuning(*P);
    if (cudaMalloc(reinterpret_cast<void **>(&P->inst), (size_t)num * sizeof(BatchInst)) != cudaSuccess) {
        delete P;
        return TL_ERROR_OUT_OF_MEMORY;
    }
    int rc = build_plan(*P, dev_offsets, st);
    if (rc) {
        cudaFree(P->inst);
        if (P->owner) cudaFree(P->owner);
        if (P->tile) cudaFree(P->tile);
        free_order_buffers(*P);
        delete P;
        return rc;
    }
    *out = reinterpret_cast<tl_batch_plan *>(P);
    return TL_SUCCESS;
}

int batch_plan_destroy(tl_batch_plan *plan) {
    if (!plan) return TL_ERROR_INVALID_VALUE;
    auto *P = reinterpret_cast<tl_batch_plan_impl *>(plan);
    cudaFree(P->inst);
    if (P->owner) cudaFree(P->owner);
    if (P->tile) cudaFree(P->tile);
    free_order_buffers(*P);
    delete P;
    return TL_SUCCESS;
}

int batch_ordered(const tl_batch_plan *plan, uint64_t *instances, uint64_t *keys) {
    if (!plan) return TL_ERROR_INVALID_VALUE;
    const auto &P = *reinterpret_cast<const tl_batch_plan_impl *>(plan);
    if (instances) *instances = P.ordered;
    if (keys) *keys = P.ordered_keys;
    return TL_SUCCESS;
}

int batch_workspace_bytes(const tl_batch_plan *plan, uint64_t *bytes) {
    if (!plan || !bytes) return TL_ERROR_INVALID_VALUE;
    *bytes = reinterpret_cast<const tl_batch_plan_impl *>(plan)->ws_bytes;
    return TL_SUCCESS;
}

template <typename K>
static int launch_batch_permute(const tl_batch_plan_impl &P, K *keys, char *ws, cudaStream_t st, int threads) {
    // every instance's scratch base shares its keys' offset within 16 bytes
    K *scr = reinterpret_cast<K *>(ws + (reinterpret_cast<uintptr_t>(keys) & 15));
    unsigned int *flags = reinterpret_cast<unsigned int *>(ws + P.off_flags);
    unsigned int *done = reinterpret_cast<unsigned int *>(ws + P.off_done);
    Ctrl *ctrl = reinterpret_cast<Ctrl *>(ws + P.off_ctrl);
    // flags, done counters and the control block are contiguous: one memset, no
    // host-to-device copy, so the launch can be captured in a CUDA graph
    TL_CUDA_TRY(cudaMemsetAsync(flags, 0, P.ws_bytes - P.off_flags, st));
    WaitCfg wc;
    wc.flag_value = 1;
    wc.wait_value = debug_force_timeout() ? 0xFFFFFFFFu : 1u;
    wc.spin_limit = debug_spin_limit();
    const size_t smem = (size_t)P.tot.max_tile * sizeof(K) + kTileSmemSlack;  // the largest tile
    auto kern = threads == 512 ? batch_permute_kernel<K, 512, kBatchBlocksPerSM512>
                               : batch_permute_kernel<K, 256, kBatchBlocksPerSM256>;
    TL_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    TL_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem));
    const uint64_t work = P.tot.tiles + P.tot.chunks;
    if (work == 0) return TL_SUCCESS;
    const uint64_t grid = std::min<uint64_t>((uint64_t)std::max(per_sm, 1) * batch_sms(), work);
    kern<<<(unsigned)grid, threads, smem, st>>>(keys, scr, P.inst, P.owner, P.tile, P.items, P.citem, P.tot, ctrl, wc,
                                                 flags, done);
    TL_CUDA_TRY(cudaGetLastError());
    return TL_SUCCESS;
}

int batch_permute(const tl_batch_plan *plan, void *dev_keys, void *dev_ws, uint64_t ws_bytes, cudaStream_t st) {
    if (!plan || !dev_keys || !dev_ws) return TL_ERROR_INVALID_VALUE;
    const auto &P = *reinterpret_cast<const tl_batch_plan_impl *>(plan);
    if (ws_bytes < P.ws_bytes) return TL_ERROR_WORKSPACE_TOO_SMALL;
    if (reinterpret_cast<uintptr_t>(dev_ws) % 256 || reinterpret_cast<uintptr_t>(dev_keys) % P.key_bytes)
        return TL_ERROR_INVALID_VALUE;
    char *ws = static_cast<char *>(dev_ws);
    return P.key_bytes == 8 ? launch_batch_permute<uint64_t>(P, static_cast<uint64_t *>(dev_keys), ws, st, P.threads)
                            : launch_batch_permute<uint32_t>(P, static_cast<uint32_t *>(dev_keys), ws, st, P.threads);
}

int batch_status(const tl_batch_plan *plan, const void *dev_ws, cudaStream_t st) {
    if (!plan || !dev_ws) return TL_ERROR_INVALID_VALUE;
    const auto &P = *reinterpret_cast<const tl_batch_plan_impl *>(plan);
    const Ctrl *ctrl = reinterpret_cast<const Ctrl *>(static_cast<const char *>(dev_ws) + P.off_ctrl);
    unsigned int err = 0;
    int rc = read_error_word(&ctrl->error, &err, st);
    if (rc) return rc;
    // a bounded wait expired, or (never expected) the ordered schedule found a
    // scratch store without scratch and skipped it
    if (!err) return TL_SUCCESS;
    return (err & (1u << TL_ERROR_TIMEOUT)) ? TL_ERROR_TIMEOUT : TL_ERROR_UNSUPPORTED;
}

int batch_query_workspace_bytes(const tl_batch_plan *plan, uint64_t q, uint64_t *bytes) {
    if (!plan || !bytes) return TL_ERROR_INVALID_VALUE;
    const auto &P = *reinterpret_cast<const tl_batch_plan_impl *>(plan);
    auto al = [](uint64_t x) { return (x + 255) / 256 * 256; };
    *bytes = al((uint64_t)P.num * 4) + al(((uint64_t)P.num + 1) * 8) + al(q * P.key_bytes) + al(q * 4) + al(q * 8);
    return TL_SUCCESS;
}

template <typename K>
static int launch_batch_query(const tl_batch_plan_impl &P, const K *keys, const K *Q, const uint32_t *qinst,
                              uint64_t q, uint64_t *ans, char *ws, cudaStream_t st) {
    auto al = [](uint64_t x) { return (x + 255) / 256 * 256; };
    unsigned int *count = reinterpret_cast<unsigned int *>(ws);
    unsigned long long *start = reinterpret_cast<unsigned long long *>(ws + al((uint64_t)P.num * 4));
    K *sq = reinterpret_cast<K *>(reinterpret_cast<char *>(start) + al(((uint64_t)P.num + 1) * 8));
    uint32_t *sinst = reinterpret_cast<uint32_t *>(reinterpret_cast<char *>(sq) + al(q * sizeof(K)));
    uint64_t *sidx = reinterpret_cast<uint64_t *>(reinterpret_cast<char *>(sinst) + al(q * 4));
    const int sms = batch_sms();
    const unsigned g = (unsigned)std::min<uint64_t>((q + 255) / 256, (uint64_t)sms * 8);
    TL_CUDA_TRY(cudaMemsetAsync(count, 0, (size_t)P.num * 4, st));
    // queries whose instance id is out of range answer 0 (their answers are
    // written here, the valid ones by the query kernel)
    TL_CUDA_TRY(cudaMemsetAsync(ans, 0, q * 8, st));
    batch_hist_kernel<<<g, 256, 0, st>>>(qinst, q, P.num, count);
    batch_scan_kernel<<<1, 1024, 0, st>>>(count, P.num, start);
    batch_bucket_kernel<K><<<g, 256, 0, st>>>(Q, qinst, q, P.num, start, sq, sinst, sidx);
    TL_CUDA_TRY(cudaGetLastError());
    // after the bucket pass start[j] holds the end of bucket j; the query kernel
    // only needs the sorted arrays.  Valid queries: start[num] (read on device).
    const uint32_t pin_cap = (uint32_t)(48 * 1024 / sizeof(K));
    const size_t smem = (size_t)pin_cap * sizeof(K);
    auto kern = batch_query_kernel<K>;
    TL_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    uint32_t *d_pin = nullptr;
    keep_pool_memory();
    TL_CUDA_TRY(cudaMallocAsync(reinterpret_cast<void **>(&d_pin), sizeof(P.pin_levels), st));
    TL_CUDA_TRY(cudaMemcpyAsync(d_pin, P.pin_levels, sizeof(P.pin_levels), cudaMemcpyHostToDevice, st));
    int per_sm = 0;
    TL_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kBatchThreads, smem));
    const uint64_t chunks = (q + P.query_chunk - 1) / P.query_chunk;
    const unsigned grid = (unsigned)std::min<uint64_t>(chunks, (uint64_t)std::max(per_sm, 1) * sms);
    kern<<<grid, kBatchThreads, smem, st>>>(keys, P.inst, sq, sinst, sidx, start + P.num, P.query_chunk, d_pin,
                                           pin_cap, ans);
    cudaFreeAsync(d_pin, st);
    TL_CUDA_TRY(cudaGetLastError());
    return TL_SUCCESS;
}

int batch_query(const tl_batch_plan *plan, const void *dev_keys, const void *dev_queries, const uint32_t *dev_inst,
                uint64_t q, uint64_t *dev_answers, void *dev_ws, uint64_t ws_bytes, cudaStream_t st, float *ms) {
    if (!plan || (q && (!dev_keys || !dev_queries || !dev_inst || !dev_answers || !dev_ws)))
        return TL_ERROR_INVALID_VALUE;
    const auto &P = *reinterpret_cast<const tl_batch_plan_impl *>(plan);
    uint64_t need = 0;
    batch_query_workspace_bytes(plan, q, &need);
    if (ws_bytes < need) return TL_ERROR_WORKSPACE_TOO_SMALL;
    if (q == 0) return TL_SUCCESS;
    EventTimer timer(ms != nullptr, st);
    timer.start();
    char *ws = static_cast<char *>(dev_ws);
    int rc = P.key_bytes == 8
                 ? launch_batch_query<uint64_t>(P, static_cast<const uint64_t *>(dev_keys),
                                                static_cast<const uint64_t *>(dev_queries), dev_inst, q, dev_answers, ws, st)
                 : launch_batch_query<uint32_t>(P, static_cast<const uint32_t *>(dev_keys),
                                                static_cast<const uint32_t *>(dev_queries), dev_inst, q, dev_answers, ws, st);
    timer.stop();
    if (rc) return rc;
    if (ms) {
        rc = sync_and_check(st);
        if (rc) return rc;
        *ms = timer.elapsed();
    }
    return TL_SUCCESS;
}

int batch_set_tuning(tl_batch_plan *plan, const uint32_t *tile_keys, const uint32_t *pin_levels, uint32_t query_chunk,
                     uint32_t threads, const int64_t *dev_offsets, cudaStream_t st) {
    if (!plan) return TL_ERROR_INVALID_VALUE;
    auto &P = *reinterpret_cast<tl_batch_plan_impl *>(plan);
    if (tile_keys) {
        for (int c = 0; c < kMaxClass; ++c) {
            const uint32_t t = tile_keys[c];
            if (t < 256 || t * P.key_bytes > 96 * 1024 || (t & (t - 1))) return TL_ERROR_INVALID_VALUE;
        }
        memcpy(P.tile_keys, tile_keys, sizeof(P.tile_keys));
        if (!dev_offsets) return TL_ERROR_INVALID_VALUE;
        int rc = build_plan(P, dev_offsets, st);
        if (rc) return rc;
    }
    if (pin_levels) memcpy(P.pin_levels, pin_levels, sizeof(P.pin_levels));
    if (query_chunk) P.query_chunk = query_chunk;
    if (threads) {
        if (threads != 256 && threads != 512) return TL_ERROR_INVALID_VALUE;
        P.threads = threads;
    }
    return TL_SUCCESS;
}

int batch_get_tuning(const tl_batch_plan *plan, uint32_t *tile_keys, uint32_t *pin_levels, uint32_t *query_chunk,
                     uint32_t *threads) {
    if (!plan) return TL_ERROR_INVALID_VALUE;
    const auto &P = *reinterpret_cast<const tl_batch_plan_impl *>(plan);
    if (tile_keys) memcpy(tile_keys, P.tile_keys, sizeof(P.tile_keys));
    if (pin_levels) memcpy(pin_levels, P.pin_levels, sizeof(P.pin_levels));
    if (query_chunk) *query_chunk = P.query_chunk;
    if (threads) *threads = P.threads;
    return TL_SUCCESS;
}

// Size classes present in the batch (floor(log2 n_j)) and the keys in each,
// read back from the plan (host).
static int batch_class_keys(const tl_batch_plan_impl &P, std::vector<uint64_t> &keys_per_class) {
    std::vector<BatchInst> h(P.num);
    TL_CUDA_TRY(cudaMemcpy(h.data(), P.inst, (size_t)P.num * sizeof(BatchInst), cudaMemcpyDeviceToHost));
    keys_per_class.assign(kMaxClass, 0);
    for (const auto &I : h) {
        const uint64_t n = I.S.g.n;
        const uint32_t c = n ? bit_length(n) - 1 : 0;
        keys_per_class[c < kMaxClass ? c : kMaxClass - 1] += n;
    }
    return TL_SUCCESS;
}

// Coordinate-descent autotuner.  Permutation: the block size, then per size class
// (largest classes first) the tile size, each candidate timed on the whole batch
// (the sorted input restored from a copy before every trial).  Queries: the
// work-item size, then per size class the number of top levels pinned in shared
// memory.  The plan keeps the best values; the keys are left sorted.
int batch_autotune(tl_batch_plan *plan, const int64_t *dev_offsets, void *dev_keys, const void *dev_queries,
                   const uint32_t *dev_inst, uint64_t q, cudaStream_t st, char *report, size_t report_len) {
    if (!plan || !dev_offsets || !dev_keys) return TL_ERROR_INVALID_VALUE;
    auto &P = *reinterpret_cast<tl_batch_plan_impl *>(plan);
    const size_t kbytes = (size_t)P.total_keys * P.key_bytes;
    char *pristine = nullptr, *ws = nullptr;
    int rc = TL_SUCCESS;
    std::vector<uint64_t> cls_keys;
    rc = batch_class_keys(P, cls_keys);
    if (rc) return rc;
    if (cudaMalloc(reinterpret_cast<void **>(&pristine), kbytes) != cudaSuccess) return TL_ERROR_OUT_OF_MEMORY;
    TL_CUDA_TRY(cudaMemcpyAsync(pristine, dev_keys, kbytes, cudaMemcpyDeviceToDevice, st));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    uint64_t ws_cap = 0;
    auto ensure_ws = [&](uint64_t need) -> int {
        if (need <= ws_cap) return TL_SUCCESS;
        if (ws) cudaFree(ws);
        ws = nullptr;
        ws_cap = 0;
        if (cudaMalloc(reinterpret_cast<void **>(&ws), need) != cudaSuccess) return TL_ERROR_OUT_OF_MEMORY;
        ws_cap = need;
        return TL_SUCCESS;
    };
    auto time_permute = [&](float &best) -> int {
        float total = 0.f;
        for (int rep = 0; rep < 3; ++rep) {
            TL_CUDA_TRY(cudaMemcpyAsync(dev_keys, pristine, kbytes, cudaMemcpyDeviceToDevice, st));
            int r = ensure_ws(P.ws_bytes);
            if (r) return r;
            cudaEventRecord(e0, st);
            r = batch_permute(plan, dev_keys, ws, ws_cap, st);
            if (r) return r;
            cudaEventRecord(e1, st);
            TL_CUDA_TRY(cudaEventSynchronize(e1));
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            if (rep) total += ms;  // first repetition warms up
        }
        best = total / 2;
        return TL_SUCCESS;
    };
    const uint32_t tiles[3] = {(uint32_t)(16384 / P.key_bytes), (uint32_t)(32768 / P.key_bytes),
                               (uint32_t)(65536 / P.key_bytes)};
    float cur = 0.f;
    rc = time_permute(cur);
    // block size
    for (uint32_t th : {512u, 256u}) {
        if (rc) break;
        const uint32_t keep = P.threads;
        P.threads = th;
        float ms = 0.f;
        rc = time_permute(ms);
        if (!rc && ms < cur) cur = ms; else P.threads = keep;
    }
    // tile size per class, largest classes first
    std::vector<int> order;
    for (int c = 0; c < kMaxClass; ++c)
        if (cls_keys[c]) order.push_back(c);
    std::sort(order.begin(), order.end(), [&](int a, int b2) { return cls_keys[a] > cls_keys[b2]; });
    for (int c : order) {
        if (rc) break;
        const uint32_t keep = P.tile_keys[c];
        uint32_t best_t = keep;
        for (uint32_t t : tiles) {
            if (t == keep) continue;
            P.tile_keys[c] = t;
            rc = build_plan(P, dev_offsets, st);
            if (rc) break;
            float ms = 0.f;
            rc = time_permute(ms);
            if (rc) break;
            if (ms < cur) {
                cur = ms;
                best_t = t;
            }
        }
        P.tile_keys[c] = best_t;
        if (!rc) rc = build_plan(P, dev_offsets, st);
    }
    float qcur = -1.f;
    if (!rc && q && dev_queries && dev_inst) {
        // a permuted copy for the query trials
        TL_CUDA_TRY(cudaMemcpyAsync(dev_keys, pristine, kbytes, cudaMemcpyDeviceToDevice, st));
        rc = ensure_ws(P.ws_bytes);
        if (!rc) rc = batch_permute(plan, dev_keys, ws, ws_cap, st);
        uint64_t qneed = 0;
        batch_query_workspace_bytes(plan, q, &qneed);
        char *qws = nullptr;
        uint64_t *ans = nullptr;
        if (!rc && (cudaMalloc(reinterpret_cast<void **>(&qws), qneed) != cudaSuccess ||
                    cudaMalloc(reinterpret_cast<void **>(&ans), q * 8) != cudaSuccess))
            rc = TL_ERROR_OUT_OF_MEMORY;
        auto time_query = [&](float &out) -> int {
            float total = 0.f;
            for (int rep = 0; rep < 3; ++rep) {
                float ms = 0.f;
                int r = batch_query(plan, dev_keys, dev_queries, dev_inst, q, ans, qws, qneed, st, &ms);
                if (r) return r;
                if (rep) total += ms;
            }
            out = total / 2;
            return TL_SUCCESS;
        };
        if (!rc) rc = time_query(qcur);
        for (uint32_t ch : {1024u, 4096u}) {
            if (rc) break;
            const uint32_t keep = P.query_chunk;
            P.query_chunk = ch;
            float ms = 0.f;
            rc = time_query(ms);
            if (!rc && ms < qcur) qcur = ms; else P.query_chunk = keep;
        }
        for (int c : order) {
            if (rc) break;
            const uint32_t keep = P.pin_levels[c];
            uint32_t best_l = keep;
            for (uint32_t L : {0u, 2u, 4u}) {
                if (L == keep) continue;
                P.pin_levels[c] = L;
                float ms = 0.f;
                rc = time_query(ms);
                if (rc) break;
                if (ms < qcur) {
                    qcur = ms;
                    best_l = L;
                }
            }
            P.pin_levels[c] = best_l;
        }
        if (qws) cudaFree(qws);
        if (ans) cudaFree(ans);
    }
    cudaMemcpyAsync(dev_keys, pristine, kbytes, cudaMemcpyDeviceToDevice, st);
    cudaStreamSynchronize(st);
    cudaFree(pristine);
    if (ws) cudaFree(ws);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (report && report_len) {
        std::string r = "{\"threads\":" + std::to_string(P.threads) + ",\"query_chunk\":" +
                        std::to_string(P.query_chunk) + ",\"permute_ms\":" + std::to_string(cur) +
                        ",\"query_ms\":" + std::to_string(qcur) + ",\"classes\":{";
        bool first = true;
        for (int c : order) {
            r += (first ? "" : ",") + std::string("\"") + std::to_string(c) + "\":{\"keys\":" +
                 std::to_string(cls_keys[c]) + ",\"tile_keys\":" + std::to_string(P.tile_keys[c]) +
                 ",\"pin_levels\":" + std::to_string(P.pin_levels[c]) + "}";
            first = false;
        }
        r += "}}";
        snprintf(report, report_len, "%s", r.c_str());
    }
    return rc;
}

}  // namespace tl
