// The reference's other algorithm families as selectable variants of the
// permutation, for ablations and as a second route to the same layouts.
//
// Built: the BST by involutions (the reference's bst-involutions family,
// gpu/src/bst-involutions.cuh:29-195, restating the published method of
// Berney and Sitchinava): every step is a self-inverse permutation applied by
// independent swaps, so each is one grid-wide launch with no scratch and no
// waits.
//  - perfect tree, n = 2^d - 1, ranks r = i + 1 in [1, 2^d - 1]: swap r with its
//    d-bit reversal, then with r's bits below its leading one reversed;
//  - otherwise (L = n - (2^h - 1) keys on the last level, which in sorted order
//    alternate with their separators at the front): unshuffle the first 2L keys
//    (leaves first) by two modular involutions (x -> x^-1 and x -> 2 x^-1 mod
//    2L - 1, after Yang, Ellis, Mamakani and Ruskey, "In-place permuting and
//    perfect shuffling using involutions"), rotate the array left by L (three
//    reversals), and lay out the 2^h - 1 front keys as a perfect tree.
// The stream permutation (permute.cu) is the library's own algorithm and the
// default; this family trades its single pass for 2-7 full passes.
#include <algorithm>

#include "internal.h"
#include "tl_common.cuh"

namespace tl {

constexpr int kVariantThreads = 256;

// r with its low `bits` bits reversed.
__device__ __forceinline__ uint64_t reverse_low_bits(uint64_t r, uint32_t bits) {
    if (bits == 0) return r;
    const uint64_t low = __brevll(r) >> (64 - bits);
    return ((r >> bits) << bits) | low;
}

template <typename K>
__device__ __forceinline__ void swap_keys(K *A, uint64_t i, uint64_t j) {
    const K t = A[i];
    A[i] = A[j];
    A[j] = t;
}

// Perfect BST, step 1: rank r <-> its d-bit reversal.
template <typename K>
__global__ void __launch_bounds__(kVariantThreads) bst_bitrev_kernel(K *A, uint64_t n, uint32_t d) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const uint64_t j = reverse_low_bits(i + 1, d) - 1;
        if (i < j) swap_keys(A, i, j);
    }
}

// Perfect BST, step 2: rank r <-> r with the bits below its leading one reversed.
template <typename K>
__global__ void __launch_bounds__(kVariantThreads) bst_lowrev_kernel(K *A, uint64_t n) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const uint64_t r = i + 1;
        const uint32_t len = 64u - (uint32_t)__clzll((long long)r);
        const uint64_t j = reverse_low_bits(r, len - 1) - 1;
        if (i < j) swap_keys(A, i, j);
    }
}

// x^-1 mod m for gcd(x, m) = 1 (extended Euclid on signed words; m < 2^63).
__device__ __forceinline__ uint64_t inverse_mod(uint64_t x, uint64_t m) {
    int64_t a = (int64_t)(x % m), b = (int64_t)m, u = 1, v = 0;
    while (b) {
        const int64_t q = a / b;
        int64_t t = a - q * b;
        a = b;
        b = t;
        t = u - q * v;
        u = v;
        v = t;
    }
    return (uint64_t)(u < 0 ? u + (int64_t)m : u);
}

__device__ __forceinline__ uint64_t gcd64(uint64_t a, uint64_t b) {
    while (b) {
        const uint64_t t = a % b;
        a = b;
        b = t;
    }
    return a;
}

// The involution x -> g * (c * (x/g)^-1 mod m/g), g = gcd(x, m), on the keys
// [1, m) of an array of m + 1 keys (the two ends stay).  c = 1 then c = 2 is the
// 2-way perfect shuffle; c = 2 then c = 1 its inverse.
template <typename K>
__global__ void __launch_bounds__(kVariantThreads) involution_kernel(K *A, uint64_t m, uint64_t c) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t x = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x + 1; x < m; x += stride) {
        const uint64_t g = gcd64(x, m), mg = m / g;
        const uint64_t y = mg > 1 ? g * ((c % mg) * inverse_mod(x / g, mg) % mg) : 0;
        if (x < y) swap_keys(A, x, y);
    }
}

// A[lo, hi) reversed.
template <typename K>
__global__ void __launch_bounds__(kVariantThreads) reverse_kernel(K *A, uint64_t lo, uint64_t hi) {
    const uint64_t half = (hi - lo) / 2, stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < half; i += stride)
        swap_keys(A, lo + i, hi - 1 - i);
}

static unsigned grid_for(uint64_t work) {
    return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((work + kVariantThreads - 1) / kVariantThreads, 148 * 16));
}

template <typename K>
static int bst_involutions(K *A, uint64_t n, cudaStream_t st) {
    uint32_t h = 0;
    while (h + 1 < 64 && (1ull << (h + 1)) <= n) ++h;  // floor(log2 n)
    uint64_t ni = n, d = h + 1;
    if (n != (1ull << (h + 1)) - 1) {
        ni = (1ull << h) - 1;
        d = h;
        const uint64_t L = n - ni;
        if (2 * L > 2) {
            involution_kernel<K><<<grid_for(2 * L), kVariantThreads, 0, st>>>(A, 2 * L - 1, 2);
            involution_kernel<K><<<grid_for(2 * L), kVariantThreads, 0, st>>>(A, 2 * L - 1, 1);
        }
        reverse_kernel<K><<<grid_for(L / 2), kVariantThreads, 0, st>>>(A, 0, L);
        reverse_kernel<K><<<grid_for((n - L) / 2), kVariantThreads, 0, st>>>(A, L, n);
        reverse_kernel<K><<<grid_for(n / 2), kVariantThreads, 0, st>>>(A, 0, n);
    }
    if (ni > 1) {
        bst_bitrev_kernel<K><<<grid_for(ni), kVariantThreads, 0, st>>>(A, ni, (uint32_t)d);
        bst_lowrev_kernel<K><<<grid_for(ni), kVariantThreads, 0, st>>>(A, ni);
    }
    TL_CUDA_TRY(cudaGetLastError());
    return TL_SUCCESS;
}

int permute_algorithm(int layout, int algorithm, void *dev_A, uint64_t n, uint64_t b, uint32_t key_bytes,
                      cudaStream_t st, float *ms) {
    if (algorithm == TL_ALGO_STREAM) return permute(layout, dev_A, n, b, key_bytes, nullptr, 0, st, ms);
    if (algorithm != TL_ALGO_INVOLUTIONS) return TL_ERROR_INVALID_VALUE;
    if (layout != TL_LAYOUT_BST) return TL_ERROR_UNSUPPORTED;  // the B-tree and vEB families are not built
    if (key_bytes != 4 && key_bytes != 8) return TL_ERROR_INVALID_VALUE;
    if (n > 0 && !dev_A) return TL_ERROR_INVALID_VALUE;
    if (reinterpret_cast<uintptr_t>(dev_A) % key_bytes) return TL_ERROR_INVALID_VALUE;
    if (n >= (1ull << 62)) return TL_ERROR_UNSUPPORTED;
    if (n <= 1) {
        if (ms) *ms = 0.f;
        return TL_SUCCESS;
    }
    EventTimer timer(ms != nullptr, st);
    timer.start();
    const int rc = key_bytes == 8 ? bst_involutions(static_cast<uint64_t *>(dev_A), n, st)
                                  : bst_involutions(static_cast<uint32_t *>(dev_A), n, st);
    timer.stop();
    if (rc) return rc;
    const int rs = sync_and_check(st);
    if (rs) return rs;
    if (ms) *ms = timer.elapsed();
    return TL_SUCCESS;
}

}  // namespace tl
