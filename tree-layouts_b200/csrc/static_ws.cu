// tl_permute_static_ws: the in-place permutation for callers that cannot
// allocate device memory.
//
// Who cannot allocate: code that runs where cudaMalloc is unavailable or not
// allowed, e.g. a plugin inside a host engine that owns every device
// allocation and hands out fixed memory budgets, or a latency-critical service
// that must not hit cudaMalloc's implicit device synchronisation or its
// failure modes in the middle of a request.  tl_permute either takes its
// workspace from the library's buffer cache (filled by cudaMalloc) or from the
// caller; this entry point
// does neither: its workspace is the fixed array below, which lives in the
// library's device image.
//
// Limits and sharing:
//  - The array is kStaticWorkspaceBytes (32 MiB) on every GPU that loads the
//    library, held until the process exits.  The permutation keeps to the
//    fixed-direction schedules (the ordered one keeps per-size tables that the
//    library would allocate); one whose workspace under them exceeds the array
//    is rejected with TL_ERROR_UNSUPPORTED before any device work.
//  - Every call uses the same array and it keeps the previous call's contents.
//    The permutation clears what must start at zero (the read flags and the
//    control block behind them, by one stream-ordered memset) on every call.
//    Calls that overlap on the GPU - on different streams, or from different
//    host threads without ordering - race on the array; callers serialise them.
//  - The first call on each device looks the array's device address up with
//    cudaGetSymbolAddress (once per device, with that device current).  Make
//    that first call before any stream capture.
//  - Like tl_permute it is synchronous: it reads the status of its bounded
//    device waits back and returns after its work on the stream has finished.
#include <mutex>

#include "internal.h"

namespace tl {

constexpr uint64_t kStaticWorkspaceBytes = 32ull << 20;

static __device__ __align__(256) unsigned char g_static_workspace[kStaticWorkspaceBytes];

constexpr int kMaxDevices = 64;
static std::once_flag g_ws_once[kMaxDevices];
static void *g_ws_ptr[kMaxDevices];
static cudaError_t g_ws_err[kMaxDevices];

// Device address of g_static_workspace on the current device (set-up on first use).
static int static_workspace(void **ptr) {
    int dev = 0;
    TL_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return TL_ERROR_UNSUPPORTED;
    std::call_once(g_ws_once[dev], [dev] {
        void *p = nullptr;
        g_ws_err[dev] = cudaGetSymbolAddress(&p, g_static_workspace);
        g_ws_ptr[dev] = p;
    });
    if (g_ws_err[dev] != cudaSuccess) {
        record_cuda_error(g_ws_err[dev]);
        return TL_ERROR_CUDA;
    }
    *ptr = g_ws_ptr[dev];
    return TL_SUCCESS;
}

}  // namespace tl

extern "C" int tl_permute_static_ws(int layout, void *dev_A, uint64_t n, uint64_t b, uint32_t key_bytes,
                                    void *stream) {
    uint64_t need = 0;
    int rc = tl::permute_workspace_bytes_fixed(layout, n, b, key_bytes, &need);
    if (rc) return rc;
    if (need > tl::kStaticWorkspaceBytes) return TL_ERROR_UNSUPPORTED;
    void *ws = nullptr;
    rc = tl::static_workspace(&ws);
    if (rc) return rc;
    // the fixed-direction schedules only: the ordered one keeps device tables
    // that the library would have to allocate
    return tl::permute(layout, dev_A, n, b, key_bytes, ws, tl::kStaticWorkspaceBytes,
                       reinterpret_cast<cudaStream_t>(stream), nullptr, nullptr, false);
}
