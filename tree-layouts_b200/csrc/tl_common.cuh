// Shared definitions for the tree-layout kernels: status codes, 64-bit division
// by a runtime-invariant divisor, small integer helpers.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/tree_layouts.h"

#define TL_HD __host__ __device__ __forceinline__

namespace tl {

// floor(x / d) for 64-bit x and an invariant divisor d >= 2, by one multiply-high
// (Granlund & Montgomery, "Division by invariant integers using multiplication",
// PLDI 1994, round-up variant): with l = ceil(log2 d) and
// m = floor(2^64 * (2^l - d) / d) + 1, q = (t + ((x - t) >> 1)) >> (l - 1) where
// t = mulhi(m, x).  Exact for every 64-bit x.
struct FastDiv64 {
    uint64_t d = 2, m = 0;
    uint32_t sh = 0;
    FastDiv64() = default;
    __host__ explicit FastDiv64(uint64_t div) : d(div) {
        uint32_t l = 0;
        while (l < 64 && ((uint64_t)1 << l) < div) ++l;
        unsigned __int128 two_l = (unsigned __int128)1 << l;
        unsigned __int128 num = (two_l - div) << 64;
        m = (uint64_t)(num / div) + 1;
        sh = l - 1;
    }
    TL_HD uint64_t div(uint64_t x) const {
#ifdef __CUDA_ARCH__
        uint64_t t = __umul64hi(m, x);
#else
        uint64_t t = (uint64_t)(((unsigned __int128)m * x) >> 64);
#endif
        return (t + ((x - t) >> 1)) >> sh;
    }
    TL_HD void divmod(uint64_t x, uint64_t &q, uint64_t &r) const {
        q = div(x);
        r = x - q * d;
    }
};

// floor(x / d) for 32-bit x and an invariant divisor 2 <= d < 2^31 (same method).
struct FastDiv32 {
    uint32_t d = 2, m = 0, sh = 0;
    FastDiv32() = default;
    __host__ explicit FastDiv32(uint32_t div) : d(div) {
        uint32_t l = 0;
        while (l < 32 && (1ull << l) < div) ++l;
        m = (uint32_t)((((1ull << l) - div) << 32) / div + 1);
        sh = l - 1;
    }
    TL_HD uint32_t div(uint32_t x) const {
#ifdef __CUDA_ARCH__
        uint32_t t = __umulhi(m, x);
#else
        uint32_t t = (uint32_t)(((uint64_t)m * x) >> 32);
#endif
        return (t + ((x - t) >> 1)) >> sh;
    }
};

TL_HD uint32_t bit_length(uint64_t x) {
#ifdef __CUDA_ARCH__
    return 64u - (uint32_t)__clzll((long long)x);
#else
    return x ? 64u - (uint32_t)__builtin_clzll(x) : 0u;
#endif
}

TL_HD uint64_t low_mask(uint32_t bits) { return bits >= 64 ? ~0ull : ((1ull << bits) - 1); }

// 32 bytes of keys in one load through the read-only path (sm_100's 256-bit
// global loads); p 32-byte aligned.
template <typename K>
__device__ __forceinline__ void ldg32(const K *p, K (&out)[32 / sizeof(K)]) {
    if constexpr (sizeof(K) == 8) {
        unsigned long long a, b, c, d;
        asm("ld.global.nc.v4.u64 {%0, %1, %2, %3}, [%4];" : "=l"(a), "=l"(b), "=l"(c), "=l"(d) : "l"(p));
        out[0] = a;
        out[1] = b;
        out[2] = c;
        out[3] = d;
    } else {
        unsigned x0, x1, x2, x3, x4, x5, x6, x7;
        asm("ld.global.nc.v8.u32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
            : "=r"(x0), "=r"(x1), "=r"(x2), "=r"(x3), "=r"(x4), "=r"(x5), "=r"(x6), "=r"(x7)
            : "l"(p));
        out[0] = x0;
        out[1] = x1;
        out[2] = x2;
        out[3] = x3;
        out[4] = x4;
        out[5] = x5;
        out[6] = x6;
        out[7] = x7;
    }
}

}  // namespace tl
