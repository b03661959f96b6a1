// The reference's other algorithm families as selectable variants of the
// permutation, for ablations and as a second route to the same layouts.
//
// Built: the BST, the B-tree and the mvEB by involutions (the reference's
// involutions family, gpu/src/bst-involutions.cuh:29-195,
// gpu/src/btree-involutions.cuh:30-168 and gpu/src/mveb-involutions.cuh:30-523,
// restating the published method of Berney and Sitchinava): every step is a
// self-inverse permutation applied by independent swaps, so each is one
// grid-wide launch with no scratch and no waits.  (mvEB: see mveb_involutions
// below.)  The cycle-leader family and the hybrid BST's last level are in
// cycles.cu; the hybrid's perfect part is bst_perfect_involutions below.
// BST:
//  - perfect tree, n = 2^d - 1, ranks r = i + 1 in [1, 2^d - 1]: swap r with its
//    d-bit reversal, then with r's bits below its leading one reversed;
//  - otherwise (L = n - (2^h - 1) keys on the last level, which in sorted order
//    alternate with their separators at the front): unshuffle the first 2L keys
//    (leaves first) by two modular involutions (x -> x^-1 and x -> 2 x^-1 mod
//    2L - 1, after Yang, Ellis, Mamakani and Ruskey, "In-place permuting and
//    perfect shuffling using involutions"), rotate the array left by L (three
//    reversals), and lay out the 2^h - 1 front keys as a perfect tree.
// B-tree, k = b + 1 (btree-involutions.cuh:30-168):
//  - perfect tree of d levels, n = k^d - 1: per level, gather every k-th key
//    (the separators) to the front in order: swap rank r = i + 1 with its d
//    base-k digits reversed, then with its low d - 1 digits reversed (a digit
//    rotation: keys by their lowest digit, the separators first), then b-way
//    shuffle the n - n/k non-separators back into order (two modular
//    involutions on n - n/k - 1); recurse on the n/k separators;
//  - otherwise (h top levels, numLeaves = n - (k^h - 1) keys below them:
//    l in full leaves, i = l / b separators between those, r = numLeaves % b
//    in the partial leaf): k-way unshuffle the first l + i keys (separators
//    last), rotate them right by i, b-way shuffle the l leaf keys back into
//    order, rotate A[i, n) right by the k^h - 1 - i remaining internal keys,
//    and lay out the k^h - 1 front keys as a perfect tree.
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

// (a b) mod m, a, b < m < 2^63.
__device__ __forceinline__ uint64_t mul_mod(uint64_t a, uint64_t b, uint64_t m) {
    if (((a | b) >> 32) == 0) return a * b % m;
    return (uint64_t)((unsigned __int128)a * b % m);
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
// [1, m) of each of `parts` arrays of m + 1 keys (the two ends stay), array p
// starting at A + p * pstride + o (o may be -1: its first key is not touched).
// c = 1 then c = k is the k-way perfect shuffle; c = k then c = 1 its inverse.
template <typename K>
__global__ void __launch_bounds__(kVariantThreads)
involution_kernel(K *A, uint64_t parts, uint64_t pstride, int64_t o, uint64_t m, uint64_t c) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x, per = m - 1, work = parts * per;
    for (uint64_t w = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; w < work; w += stride) {
        const uint64_t p = w / per, x = w - p * per + 1;
        const uint64_t g = gcd64(x, m), mg = m / g;
        const uint64_t y = mg > 1 ? g * mul_mod(c % mg, inverse_mod(x / g, mg), mg) : 0;
        if (x < y) {
            K *a = A + (int64_t)(p * pstride) + o;
            swap_keys(a, x, y);
        }
    }
}

// A[lo, hi) reversed.
template <typename K>
__global__ void __launch_bounds__(kVariantThreads) reverse_kernel(K *A, uint64_t lo, uint64_t hi) {
    const uint64_t half = (hi - lo) / 2, stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < half; i += stride)
        swap_keys(A, lo + i, hi - 1 - i);
}

// Perfect B-tree level step: rank r = i + 1 (d base-k digits) <-> r with its
// low `low` digits reversed (kl = k^low).
template <typename K>
__global__ void __launch_bounds__(kVariantThreads)
digit_reverse_kernel(K *A, uint64_t n, FastDiv64 fk, uint32_t low, uint64_t kl) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        uint64_t x = i + 1, rev = 0;
        for (uint32_t t = 0; t < low; ++t) {
            uint64_t q, dg;
            fk.divmod(x, q, dg);
            rev = rev * fk.d + dg;
            x = q;
        }
        const uint64_t j = x * kl + rev - 1;
        if (i < j) swap_keys(A, i, j);
    }
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
            involution_kernel<K><<<grid_for(2 * L), kVariantThreads, 0, st>>>(A, 1, 0, 0, 2 * L - 1, 2);
            involution_kernel<K><<<grid_for(2 * L), kVariantThreads, 0, st>>>(A, 1, 0, 0, 2 * L - 1, 1);
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

// The perfect BST of ni = 2^d - 1 front keys by its two involutions (the
// hybrid BST's second part, gpu/src/bst-hybrid.cuh:93-112).
template <typename K>
static int bst_perfect_involutions(K *A, uint64_t ni, cudaStream_t st) {
    if (ni <= 1) return TL_SUCCESS;
    uint32_t d = 0;
    while ((1ull << d) <= ni) ++d;
    bst_bitrev_kernel<K><<<grid_for(ni), kVariantThreads, 0, st>>>(A, ni, d);
    bst_lowrev_kernel<K><<<grid_for(ni), kVariantThreads, 0, st>>>(A, ni);
    TL_CUDA_TRY(cudaGetLastError());
    return TL_SUCCESS;
}

// k-way shuffle (the N / k keys of each residue class interleaved back) and
// its inverse, N a multiple of k: two modular involutions on [1, N - 1).  On
// `parts` arrays of N keys at A + p * pstride + o (o = -1: an array that
// starts one key before A, whose first key the involutions never touch).
template <typename K>
static void kway_shuffle(K *A, uint64_t N, uint64_t k, bool inverse, cudaStream_t st, uint64_t parts = 1,
                         uint64_t pstride = 0, int64_t o = 0) {
    if (N <= 2 || k <= 1 || parts == 0) return;
    const uint64_t c0 = inverse ? k : 1, c1 = inverse ? 1 : k;
    involution_kernel<K><<<grid_for(parts * N), kVariantThreads, 0, st>>>(A, parts, pstride, o, N - 1, c0);
    involution_kernel<K><<<grid_for(parts * N), kVariantThreads, 0, st>>>(A, parts, pstride, o, N - 1, c1);
}

// A[lo, hi) rotated right by s (three reversals).
template <typename K>
static void rotate_right(K *A, uint64_t lo, uint64_t hi, uint64_t s, cudaStream_t st) {
    if (s == 0 || s >= hi - lo) return;
    reverse_kernel<K><<<grid_for((hi - lo) / 2), kVariantThreads, 0, st>>>(A, lo, hi);
    reverse_kernel<K><<<grid_for(s / 2), kVariantThreads, 0, st>>>(A, lo, lo + s);
    reverse_kernel<K><<<grid_for((hi - lo - s) / 2), kVariantThreads, 0, st>>>(A, lo + s, hi);
}

template <typename K>
static void btree_perfect_involutions(K *A, uint64_t n, uint64_t b, uint32_t d, cudaStream_t st) {
    const uint64_t k = b + 1;
    const FastDiv64 fk(k);
    while (d > 1) {
        uint64_t kd1 = 1;  // k^(d-1)
        for (uint32_t t = 0; t + 1 < d; ++t) kd1 *= k;
        // all d digits (nothing above them: kl unused), then the low d - 1
        digit_reverse_kernel<K><<<grid_for(n), kVariantThreads, 0, st>>>(A, n, fk, d, 0);
        digit_reverse_kernel<K><<<grid_for(n), kVariantThreads, 0, st>>>(A, n, fk, d - 1, kd1);
        kway_shuffle(A + n / k, kd1 * b, b, false, st);
        n /= k;
        --d;
    }
}

template <typename K>
static int btree_involutions(K *A, uint64_t n, uint64_t b, cudaStream_t st) {
    const uint64_t k = b + 1;
    uint32_t d = 0;  // levels of the largest perfect tree within n keys
    uint64_t pw = 1;
    while (pw <= (n + 1) / k) {
        pw *= k;
        ++d;
    }
    const uint64_t ni = pw - 1;
    if (ni != n) {
        const uint64_t nl = n - ni, l = nl - nl % b, i = l / b;
        kway_shuffle(A, l + i, k, true, st);
        rotate_right(A, 0, l + i, i, st);
        kway_shuffle(A + i, l, b, false, st);
        rotate_right(A, i, n, ni - i, st);
    }
    btree_perfect_involutions(A, ni, b, d, st);
    TL_CUDA_TRY(cudaGetLastError());
    return TL_SUCCESS;
}

// Balanced mvEB step on each array of m = kk^2 - 1 keys in A[0, total): rank
// r = i + 1 = x1 kk + x0 <-> x0 kk + x1 (the 2-digit base-kk reversal: the
// kk - 1 root keys to the front, then the keys by their lowest digit).
template <typename K>
__global__ void __launch_bounds__(kVariantThreads) digit_swap_kernel(K *A, uint64_t total, uint64_t m, uint64_t kk) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; g < total; g += stride) {
        const uint64_t p = g / m, i = g - p * m, r = i + 1;
        const uint64_t x1 = r / kk, x0 = r - x1 * kk, j = x0 * kk + x1 - 1;
        if (i < j) swap_keys(A + p * m, i, j);
    }
}

__host__ static bool is_pow2(uint64_t x) { return (x & (x - 1)) == 0; }

// The modified vEB split of a d-level tree: root_d + leaf_d = d, leaf_d the
// power of two at or above ceil((d - 2) / 2) + 1 (gpu/src/mveb-involutions.cuh:
// 257-266).
__host__ static void mveb_split(uint32_t d, uint32_t &root_d, uint32_t &leaf_d) {
    root_d = (d - 2) / 2 + 1;
    leaf_d = d - root_d;
    if (!is_pow2(leaf_d)) {
        uint32_t p = 1;
        while (p < leaf_d) p <<= 1;
        leaf_d = p;
        root_d = d - leaf_d;
    }
}

// Every array of m = 2^d - 1 keys (d a power of two) in A[0, total) into mvEB:
// per round, each array's sqrt(m + 1) - 1 root keys to its front and its
// bottoms back into order, then the round on arrays of that size.
template <typename K>
static void mveb_balanced(K *A, uint64_t total, uint64_t m, uint32_t d, cudaStream_t st) {
    while (d > 1 && total) {
        const uint64_t k = (1ull << (d / 2)) - 1;
        digit_swap_kernel<K><<<grid_for(total), kVariantThreads, 0, st>>>(A, total, m, k + 1);
        kway_shuffle(A + k, m - k, k, false, st, total / m, m);
        m = k;
        d /= 2;
    }
}

// A perfect tree of n = 2^d - 1 keys into mvEB: its root keys (every
// (l + 1)-th) to the front by a (l + 1)-way unshuffle of the n + 1 keys from
// A - 1, its bottoms back into order by an l-way shuffle; then the bottoms
// (balanced) and the root.
template <typename K>
static void mveb_perfect(K *A, uint64_t n, uint32_t d, cudaStream_t st) {
    if (n <= 1) return;
    if (is_pow2(d)) return mveb_balanced(A, n, n, d, st);
    uint32_t rd, ld;
    mveb_split(d, rd, ld);
    const uint64_t r = (1ull << rd) - 1, l = (1ull << ld) - 1;
    kway_shuffle(A, n + 1, l + 1, true, st, 1, 0, -1);
    kway_shuffle(A + r, n - r, l, false, st);
    mveb_balanced(A + r, n - r, l, ld, st);
    mveb_perfect(A, r, rd, st);
}

// Any n (gpu/src/mveb-involutions.cuh:350-497): the root keys between full
// bottoms to the front (unshuffle, rotation, shuffle), the root keys beyond
// them after those (rotation); the root and full bottoms as perfect trees, the
// incomplete bottom at the end recursively.
template <typename K>
static void mveb_involutions(K *A, uint64_t n, cudaStream_t st) {
    if (n <= 1) return;
    uint32_t d = 0;
    while (d < 63 && (1ull << d) <= n) ++d;  // bit length
    if (n == (1ull << d) - 1) return mveb_perfect(A, n, d, st);
    uint32_t rd, ld;
    mveb_split(d, rd, ld);
    const uint64_t r = (1ull << rd) - 1, l = (1ull << ld) - 1;
    const uint64_t nf = (n - r) / l, inc = n - r - nf * l, tn = nf * (l + 1);
    kway_shuffle(A, tn, l + 1, true, st);
    rotate_right(A, 0, tn, nf, st);
    kway_shuffle(A + nf, tn - nf, l, false, st);
    if (nf < r) rotate_right(A, nf, n, r - nf, st);
    if (rd == ld) {
        mveb_balanced(A, n - inc, r, rd, st);
    } else {
        mveb_balanced(A + r, nf * l, l, ld, st);
        mveb_perfect(A, r, rd, st);
    }
    mveb_involutions(A + (n - inc), inc, st);
}

template <typename K>
static int mveb_involutions_run(K *A, uint64_t n, cudaStream_t st) {
    mveb_involutions(A, n, st);
    TL_CUDA_TRY(cudaGetLastError());
    return TL_SUCCESS;
}

int permute_algorithm(int layout, int algorithm, void *dev_A, uint64_t n, uint64_t b, uint32_t key_bytes,
                      cudaStream_t st, float *ms) {
    if (algorithm == TL_ALGO_STREAM) return permute(layout, dev_A, n, b, key_bytes, nullptr, 0, st, ms);
    if (algorithm < TL_ALGO_INVOLUTIONS || algorithm > TL_ALGO_HYBRID) return TL_ERROR_INVALID_VALUE;
    if (layout < TL_LAYOUT_BST || layout > TL_LAYOUT_VEB) return TL_ERROR_INVALID_VALUE;
    if (layout == TL_LAYOUT_VEB) return TL_ERROR_UNSUPPORTED;  // the reference has it on the CPU only
    if (algorithm == TL_ALGO_HYBRID && layout != TL_LAYOUT_BST) return TL_ERROR_UNSUPPORTED;
    if (layout == TL_LAYOUT_BTREE && (b == 0 || b >= (1ull << 31))) return TL_ERROR_INVALID_VALUE;
    if (algorithm == TL_ALGO_CYCLES && layout == TL_LAYOUT_BTREE && b >= (1ull << 20)) return TL_ERROR_UNSUPPORTED;
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
    int rc = TL_SUCCESS;
    if (algorithm == TL_ALGO_CYCLES) {
        rc = permute_cycles(layout, algorithm, dev_A, n, b, key_bytes, st, nullptr);
    } else if (algorithm == TL_ALGO_HYBRID) {
        uint64_t ni = 0;
        rc = permute_cycles(layout, algorithm, dev_A, n, b, key_bytes, st, &ni);
        if (!rc)
            rc = key_bytes == 8 ? bst_perfect_involutions(static_cast<uint64_t *>(dev_A), ni, st)
                                : bst_perfect_involutions(static_cast<uint32_t *>(dev_A), ni, st);
    } else if (layout == TL_LAYOUT_BST) {
        rc = key_bytes == 8 ? bst_involutions(static_cast<uint64_t *>(dev_A), n, st)
                            : bst_involutions(static_cast<uint32_t *>(dev_A), n, st);
    } else if (layout == TL_LAYOUT_BTREE) {
        rc = key_bytes == 8 ? btree_involutions(static_cast<uint64_t *>(dev_A), n, b, st)
                            : btree_involutions(static_cast<uint32_t *>(dev_A), n, b, st);
    } else {
        rc = key_bytes == 8 ? mveb_involutions_run(static_cast<uint64_t *>(dev_A), n, st)
                            : mveb_involutions_run(static_cast<uint32_t *>(dev_A), n, st);
    }
    timer.stop();
    if (rc) return rc;
    const int rs = sync_and_check(st);
    if (rs) return rs;
    if (ms) *ms = timer.elapsed();
    return TL_SUCCESS;
}

}  // namespace tl
