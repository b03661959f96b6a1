// mvEB / standard vEB streaming permutation: the unit tables and the per-tile
// helpers over a MvebPlan (geometry.cuh), shared by the permutation, its host
// replay and the reverse permutation.
#pragma once

#include "geometry.cuh"

namespace tl {

// Unit tables: for a unit of U levels (1 <= U <= 8), inv[unit_table_off(U) + q]
// is the sorted rank (within the unit) held at unit position q.
TL_HD uint32_t unit_table_off(uint32_t U) { return (1u << U) - U - 1; }  // sum of 2^u - 1 over u < U
constexpr uint32_t kUnitTableBytes = (1u << 9) - 9 - 1;                   // unit_table_off(9)

struct MvebParams {
    MvebPlan plan;
    unsigned char inv[kUnitTableBytes];
};

TL_HD int mveb_region_of_tile(const MvebPlan &P, uint64_t k) {
    int r = 0;
    while (r + 1 < P.nreg && k >= P.reg[r + 1].tile_base) ++r;
    return r;
}

TL_HD uint64_t mveb_tile_of(const MvebPlan &P, uint64_t x) {
    int r = 0;
    while (r + 1 < P.nreg && x >= P.reg[r + 1].src) ++r;
    const MvebRegion &R = P.reg[r];
    return R.tile_base + (x - R.src) / R.tile_len;
}

TL_HD void mveb_tile(const MvebPlan &P, uint64_t k, int &ri, uint64_t &p0, uint64_t &p1) {
    ri = mveb_region_of_tile(P, k);
    const MvebRegion &R = P.reg[ri];
    p0 = R.src + (k - R.tile_base) * R.tile_len;
    p1 = R.src + R.len < p0 + R.tile_len ? R.src + R.len : p0 + R.tile_len;
}

// Groups [g0, g1) of a unit-region tile; the last group of a perfect segment has
// no separator.
TL_HD void mveb_tile_groups(const MvebRegion &R, uint64_t p0, uint64_t p1, uint64_t &g0, uint64_t &g1) {
    const uint64_t u = (1ull << R.U) - 1;
    g0 = (p0 - R.src) >> R.U;
    g1 = (p1 - R.src + u) >> R.U;
}

TL_HD bool mveb_tile_wait(const MvebPlan &P, const MvebRegion &R, uint64_t p0, uint64_t p1, uint64_t &k_lo,
                          uint64_t &k_hi) {
    if (R.U == 0) return false;
    uint64_t g0, g1;
    mveb_tile_groups(R, p0, p1, g0, g1);
    const uint64_t d0 = mveb_unit_dst(R, g0);
    const uint64_t d1 = mveb_unit_dst(R, g1 - 1) + (1ull << R.U) - 1;
    const uint64_t lo = d0 > p1 ? d0 : p1;
    if (lo >= d1) return false;
    k_lo = mveb_tile_of(P, lo);
    k_hi = mveb_tile_of(P, d1 - 1);
    return true;
}

// Sorted rank held by scratch slot s, or ~0 for an unused slot.
TL_HD uint64_t mveb_slot_rank(const MvebPlan &P, uint64_t s) {
    int r = 0;
    while (r + 1 < P.nreg && s >= P.reg[r + 1].slot_base) ++r;
    const MvebRegion &R = P.reg[r];
    const uint64_t rank =
        R.U ? R.src + ((s - R.slot_base) << R.U) + ((1ull << R.U) - 1) : R.src + (s - R.slot_base);
    return rank < R.src + R.len ? rank : ~0ull;
}

inline void fill_unit_tables(MvebParams &prm) {
    const bool modified = prm.plan.modified != 0;
    for (uint32_t U = 1; U <= 8; ++U) {
        unsigned char *inv = prm.inv + unit_table_off(U);
        const uint64_t m = (1ull << U) - 1;
        for (uint64_t s = 0; s < m; ++s) inv[veb_pos(m, s, modified)] = (unsigned char)s;
    }
}

}  // namespace tl
