// Workspaces of the library's synchronous calls (tl_permute, tl_unpermute,
// and the algorithm variants when the caller passes none).
//
// Each call holds a device buffer only while it runs: these calls return after
// their work on the stream has finished.  The buffers are kept per device and
// reused, and new ones come from cudaMalloc: on B200 a first stream-ordered
// allocation of 250 MB took 27 ms (the pool maps its memory on growth) where
// cudaMalloc took 0.5 ms, and a permutation of 5e8 keys takes 1.4 ms.
#include <mutex>
#include <vector>

#include "internal.h"

namespace tl {

namespace {
struct CachedBuffer {
    void *p;
    size_t bytes;
    int dev;
    bool busy;
};
constexpr size_t kMaxCachedBuffers = 8;  // per process; a busy buffer is never evicted
std::mutex g_ws_mu;
std::vector<CachedBuffer> g_ws;
}  // namespace

void *workspace_acquire(size_t bytes) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    std::lock_guard<std::mutex> lk(g_ws_mu);
    CachedBuffer *best = nullptr;
    for (auto &b : g_ws)
        if (!b.busy && b.dev == dev && b.bytes >= bytes && (!best || b.bytes < best->bytes)) best = &b;
    if (best) {
        best->busy = true;
        return best->p;
    }
    // room for a new buffer: drop the smallest idle one of this device if full
    if (g_ws.size() >= kMaxCachedBuffers) {
        size_t k = g_ws.size();
        for (size_t j = 0; j < g_ws.size(); ++j)
            if (!g_ws[j].busy && g_ws[j].dev == dev && (k == g_ws.size() || g_ws[j].bytes < g_ws[k].bytes)) k = j;
        if (k == g_ws.size()) return nullptr;  // every cached buffer is in use
        cudaFree(g_ws[k].p);
        g_ws.erase(g_ws.begin() + (long)k);
    }
    void *p = nullptr;
    if (cudaMalloc(&p, bytes) != cudaSuccess) {
        cudaGetLastError();
        // an idle smaller buffer of this device may be what keeps memory short
        for (size_t j = 0; j < g_ws.size(); ++j)
            if (!g_ws[j].busy && g_ws[j].dev == dev) {
                cudaFree(g_ws[j].p);
                g_ws.erase(g_ws.begin() + (long)j);
                --j;
            }
        if (cudaMalloc(&p, bytes) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
    }
    g_ws.push_back(CachedBuffer{p, bytes, dev, true});
    return p;
}

// The library's stream-ordered allocations (query partitions, batched plans,
// rank-model training, and workspaces the cache cannot provide) come from the
// device's default pool; keep freed blocks in the pool instead of returning
// them to the driver at every synchronisation, so repeated calls reuse them
// without re-mapping memory (a 250 MB re-map took 27 to 79 ms on B200).
void keep_pool_memory() {
    static std::once_flag once[64];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
        cudaGetLastError();
        return;
    }
    std::call_once(once[dev], [dev] {
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
            uint64_t keep = UINT64_MAX;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        }
        cudaGetLastError();
    });
}

void workspace_release(void *p) {
    std::lock_guard<std::mutex> lk(g_ws_mu);
    for (auto &b : g_ws)
        if (b.p == p) b.busy = false;
}

}  // namespace tl
