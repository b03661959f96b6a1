// Building blocks of the in-place streaming permutation: the per-launch control
// block, tile tickets, read-done flags with bounded waits, and the tile loader.
//
// The in-place pass walks the array one tile at a time.  Tiles are handed out by
// an atomic ticket counter, so a CTA holding ticket t knows every ticket below t
// is already owned by a running CTA.  A CTA first copies its whole source tile
// into shared memory and then publishes "tile read".  Before storing, it waits
// (acquire) for the flags of the tiles whose source overlaps the destinations
// it will write.  Those tiles always hold smaller tickets, and a CTA publishes
// its flag before it waits on anything, so every wait ends.  Waits
// are still bounded: on expiry the CTA records TL_ERROR_TIMEOUT in the control
// block, skips its stores, and the host reports the error.
#pragma once

#include "tl_common.cuh"

namespace tl {

// Per-launch control block in device memory: zeroed (one memset) before each
// launch, so a launch needs no host-to-device copy and can be captured in a graph.
struct Ctrl {
    unsigned long long ticket;
    unsigned int error;
    unsigned int pad0;
    unsigned long long stalled_waits;  // waits whose flag was not set at the first look
    unsigned long long stall_polls;    // polls those waits took
    unsigned int pad[8];
};

// Wait parameters, passed to the kernels by value.
struct WaitCfg {
    unsigned int flag_value;  // value a tile publishes once its source is read
    unsigned int wait_value;  // value a wait expects (== flag_value except in fault tests)
    unsigned int spin_limit;  // iterations of a bounded wait (x ~256 ns each)
};

__device__ __forceinline__ unsigned int ld_acquire(const unsigned int *p) {
    unsigned int v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_relaxed(unsigned int *p, unsigned int v) {
    asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Waits until flag == want; false (and the error recorded) if the bound expires.
__device__ __forceinline__ bool wait_flag(const unsigned int *flag, unsigned int want, Ctrl *ctrl,
                                          const WaitCfg &wc) {
    unsigned int limit = wc.spin_limit;
    unsigned int ns = 32;
    for (unsigned int it = 0; it <= limit; ++it) {
        if (ld_acquire(flag) == want) {
            if (it) {
                atomicAdd(&ctrl->stalled_waits, 1ull);
                atomicAdd(&ctrl->stall_polls, (unsigned long long)it);
            }
            return true;
        }
        __nanosleep(ns);
        if (ns < 256) ns <<= 1;
    }
    atomicOr(&ctrl->error, 1u << TL_ERROR_TIMEOUT);
    return false;
}

// Block-wide: publish that this tile's source has been read into shared memory.
// Every load of the tile has returned its data (cp.async.wait_all, or register
// loads already stored to shared memory) before the barrier, so no write that
// follows the flag can reach them: a relaxed store suffices, and thread 0 does
// not wait for its own earlier global stores to drain as a fence would make it.
__device__ __forceinline__ void publish_read(unsigned int *flag, const WaitCfg &wc) {
    __syncthreads();
    if (threadIdx.x == 0) st_relaxed(flag, wc.flag_value);
}

// Block-wide ticket loop with the next ticket claimed one tile ahead: thread 0
// issues the atomic for ticket t+1 before tile t is processed and publishes it
// after.  A block holds at most its current and its next ticket; the current
// tile only ever waits on smaller tickets, all of them claimed earlier, so the
// smallest unfinished current tile always progresses.
struct TicketPipe {
    unsigned long long next;
};

__device__ __forceinline__ unsigned long long ticket_first(Ctrl *ctrl, unsigned long long *s_ticket) {
    if (threadIdx.x == 0) *s_ticket = atomicAdd(&ctrl->ticket, 1ull);
    __syncthreads();
    return *s_ticket;
}

__device__ __forceinline__ void ticket_claim(Ctrl *ctrl, TicketPipe &tp) {
    if (threadIdx.x == 0) tp.next = atomicAdd(&ctrl->ticket, 1ull);
}

__device__ __forceinline__ unsigned long long ticket_advance(const TicketPipe &tp, unsigned long long *s_ticket) {
    __syncthreads();  // the block is done with the current tile
    if (threadIdx.x == 0) *s_ticket = tp.next;
    __syncthreads();
    return *s_ticket;
}

// Bytes of dynamic shared memory a tile kernel asks for beyond its tile: room
// to start the buffer on a 128-byte line, and the tile's head of up to 128
// bytes (see load_tile_issue).
constexpr size_t kTileSmemSlack = 128 + 128;

// The tile buffer of a tile kernel: its dynamic shared memory rounded up to a
// 128-byte line (whatever the static shared memory before it).
template <typename K>
__device__ __forceinline__ K *tile_smem(unsigned char *dyn) {
    return reinterpret_cast<K *>((reinterpret_cast<uintptr_t>(dyn) + 127) & ~(uintptr_t)127);
}

// The base of load_tile for a tile starting at p0: p0 rounded down to a
// Line-byte boundary of the global address (Line = 128 for a buffer from
// tile_smem, 16 for one that keeps its own placement).
template <uint32_t Line = 128, typename K>
__device__ __forceinline__ uint64_t tile_base(const K *src, uint64_t p0) {
    return p0 - (reinterpret_cast<uintptr_t>(src + p0) & (Line - 1)) / sizeof(K);
}

// Copies src[p0, p1) into shared memory so that element x sits at
// sm[x - base], base = tile_base<Line>(src, p0).  With Line = 128 and a
// line-aligned buffer the copy keeps each key's offset within its 128-byte
// line, so a warp's 16-byte cp.async chunks (global -> shared without
// registers, every thread with all of its copies in flight) fill whole sectors
// on both sides; shifted against the line, each chunk fetches its own 32-byte
// sector, twice the L2 traffic.  (The vEB stream kernel measured faster with
// its buffer where the static shared memory leaves it and Line = 16.)  The
// ragged ends use plain loads.  In two halves: issue returns base with the
// interior's copies still in flight, load_tile_wait waits for them.  Threads
// tid of nt (default: the whole block) share the copies.
template <uint32_t Line = 128, typename K>
__device__ __forceinline__ uint64_t load_tile_issue(const K *__restrict__ src, uint64_t p0, uint64_t p1, K *sm,
                                                    uint32_t tid = threadIdx.x, uint32_t nt = blockDim.x) {
    constexpr uint32_t V = 16 / sizeof(K);
    const uintptr_t addr0 = reinterpret_cast<uintptr_t>(src + p0);
    const uint64_t base = tile_base<Line>(src, p0);
    const uint64_t head = (addr0 & 15) / sizeof(K);  // elements before the 16-byte boundary
    uint64_t a0 = head ? p0 + (V - head) : p0;      // first aligned element
    if (a0 > p1) a0 = p1;
    const uint64_t nvec = (p1 - a0) / V;
    const uint64_t a1 = a0 + nvec * V;
    for (uint64_t x = p0 + tid; x < a0; x += nt) sm[x - base] = src[x];
    const char *gsrc = reinterpret_cast<const char *>(src + a0);
    const uint32_t sdst = (uint32_t)__cvta_generic_to_shared(sm + (a0 - base));
    for (uint64_t v = tid; v < nvec; v += nt)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(sdst + (uint32_t)(v * 16)),
                     "l"(gsrc + v * 16)
                     : "memory");
    for (uint64_t x = a1 + tid; x < p1; x += nt) sm[x - base] = src[x];
    return base;
}

__device__ __forceinline__ void load_tile_wait() { asm volatile("cp.async.wait_all;" ::: "memory"); }

template <uint32_t Line = 128, typename K>
__device__ __forceinline__ uint64_t load_tile(const K *__restrict__ src, uint64_t p0, uint64_t p1, K *sm) {
    const uint64_t base = load_tile_issue<Line>(src, p0, p1, sm);
    load_tile_wait();
    return base;
}

}  // namespace tl
