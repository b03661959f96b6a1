// Global -> shared -> global copies with the bulk-copy engine (cp.async.bulk,
// sm_90+): one elected thread per CTA keeps a ring of shared-memory stages
// moving; loads complete on an mbarrier (transaction bytes), stores are
// committed as bulk groups and waited on before a stage is refilled.  Used for
// the B-tree permutation's second pass, a plain copy of the scratch ranges.
//
// Every wait is bounded: on expiry the kernel records TL_ERROR_TIMEOUT and
// stops issuing; before returning it waits (again bounded) for the copies it
// has in flight.  The bound is fixed (about a quarter of a second per wait,
// far above a real copy's microseconds) and does not follow the test hook
// that shortens the read-flag waits: these waits never depend on another CTA.
#pragma once

#include "stream.cuh"

namespace tl {

constexpr int kBulkStages = 6;           // shared-memory stages per CTA
constexpr int kBulkAhead = 4;            // loads in flight ahead of the store (stages - 2)
constexpr uint32_t kBulkChunk = 16384;   // bytes per stage
constexpr int kMaxBulkRanges = 48;
constexpr unsigned int kBulkSpinLimit = 1u << 22;  // x (try_wait + 64 ns)
static_assert(kBulkStages - kBulkAhead == 2, "a refilled stage was last stored two chunks ago");

// One copy range split for the bulk engine: its 16-byte-aligned interior
// (byte offsets into the destination and source arrays, a multiple of 16 bytes
// long) and the ragged keys before and after it.
struct BulkRange {
    uint64_t dst, src, bytes;   // interior, in bytes from the array starts
    uint64_t chunk0;            // first chunk of the interior in the plan's numbering
    uint64_t key_dst, key_src;  // first key of the range (ragged ends are copied by key)
    uint32_t head, tail;        // keys before / after the interior
    uint64_t len;               // keys of the range
};

struct BulkPlan {
    int nr;
    uint64_t nchunks;
    BulkRange r[kMaxBulkRanges];
};

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait for phase `parity` of an mbarrier.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
    for (unsigned int it = 0; it <= kBulkSpinLimit; ++it) {
        if (mbar_try_wait(bar, parity)) return true;
        __nanosleep(64);
    }
    return false;
}

__device__ __forceinline__ void bulk_load(void *smem_dst, const void *gsrc, uint32_t bytes, uint64_t *bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(smem_dst)),
                 "l"(gsrc), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void bulk_store(void *gdst, const void *smem_src, uint32_t bytes) {
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(gdst), "r"(smem_u32(smem_src)),
                 "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_read2() { asm volatile("cp.async.bulk.wait_group.read 2;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

// Chunk k of this CTA (global chunk blockIdx.x + k * gridDim.x): its range,
// found with a cursor that only moves forward as k grows.
struct BulkCursor {
    int r = 0;
    __device__ __forceinline__ void seek(const BulkPlan &P, uint64_t c) {
        while (r + 1 < P.nr && c >= P.r[r + 1].chunk0) ++r;
    }
};

// Copies the plan's ranges from `src` to `dst` (byte arrays).  One warp per
// CTA: lane 0 drives the bulk engine, the other lanes of CTA 0 copy the
// ragged keys.  `stage` is kBulkStages * kBulkChunk bytes of shared memory,
// 128-byte aligned.
template <typename K>
__device__ __forceinline__ void bulk_copy_plan(K *dst, const K *src, const BulkPlan &P, unsigned char *stage,
                                               uint64_t *bars, Ctrl *ctrl) {
    if (blockIdx.x == 0 && threadIdx.x > 0) {  // ragged ends, key by key
        for (int j = 0; j < P.nr; ++j) {
            const BulkRange &R = P.r[j];
            for (uint32_t e = threadIdx.x - 1; e < R.head + R.tail; e += blockDim.x - 1) {
                const uint64_t o = e < R.head ? e : R.len - R.tail + (e - R.head);
                dst[R.key_dst + o] = src[R.key_src + o];
            }
        }
    }
    if (threadIdx.x != 0) return;
    char *gd = reinterpret_cast<char *>(dst);
    const char *gs = reinterpret_cast<const char *>(src);
    for (int s = 0; s < kBulkStages; ++s) mbar_init(&bars[s], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    const uint64_t mine = P.nchunks > blockIdx.x ? (P.nchunks - 1 - blockIdx.x) / gridDim.x + 1 : 0;
    BulkCursor lc, sc;
    auto load = [&](uint64_t k) {
        const uint64_t c = blockIdx.x + k * gridDim.x;
        lc.seek(P, c);
        const BulkRange &R = P.r[lc.r];
        const uint64_t off = (c - R.chunk0) * kBulkChunk;
        const uint32_t bytes = (uint32_t)min((uint64_t)kBulkChunk, R.bytes - off);
        const int s = (int)(k % kBulkStages);
        mbar_expect_tx(&bars[s], bytes);
        bulk_load(stage + (size_t)s * kBulkChunk, gs + R.src + off, bytes, &bars[s]);
    };
    uint64_t k = 0;
    for (; k < mine && k < (uint64_t)kBulkAhead; ++k) load(k);
    bool ok = true;
    uint64_t issued = k;  // loads issued
    for (k = 0; k < mine; ++k) {
        const int s = (int)(k % kBulkStages);
        if (!mbar_wait(&bars[s], (uint32_t)((k / kBulkStages) & 1))) {
            ok = false;
            break;
        }
        const uint64_t c = blockIdx.x + k * gridDim.x;
        sc.seek(P, c);
        const BulkRange &R = P.r[sc.r];
        const uint64_t off = (c - R.chunk0) * kBulkChunk;
        const uint32_t bytes = (uint32_t)min((uint64_t)kBulkChunk, R.bytes - off);
        bulk_store(gd + R.dst + off, stage + (size_t)s * kBulkChunk, bytes);
        bulk_commit();
        if (issued < mine) {
            bulk_wait_read2();  // the stage of chunk issued - kBulkStages = k - 2 has been read out
            load(issued++);
        }
    }
    if (!ok) {
        atomicOr(&ctrl->error, 1u << TL_ERROR_TIMEOUT);
        // loads still in flight land in shared memory: wait for them (bounded)
        for (uint64_t j = k; j < issued; ++j)
            mbar_wait(&bars[j % kBulkStages], (uint32_t)((j / kBulkStages) & 1));
    }
    bulk_wait_all();
}

}  // namespace tl
