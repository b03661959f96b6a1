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

}  // namespace tl
