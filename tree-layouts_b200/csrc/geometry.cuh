// Layout geometry shared by host and device: where sorted rank s lands in each
// implicit layout, and the host-side plans the permutation kernels execute.
//
// Level-order B-tree (b keys per node; the BST is b = 1).  Node k holds positions
// [k*b, k*b + b) and its children are nodes k*(b+1)+1 .. k*(b+1)+b+1
// (gpu/src/query-btree.cuh:51).  With h = floor(log_{b+1} n) the top h levels form
// a perfect tree of ni = (b+1)^h - 1 keys; the last level holds the remaining
// nl = n - ni keys in i = (nl - nl % b)/b full leaves plus one partial leaf of
// r = nl % b keys (cpu/src/btree-cycles.h:32-39, gpu/src/btree-cycles.cuh:32-60).
// In sorted order the first l + i keys (l = i*b) alternate b leaf keys and one
// separator; then come the r partial-leaf keys; then the remaining top keys.
//
// Modified van Emde Boas (gpu/src/mveb-cycles.cuh): a tree of d = bitlen(n)
// levels splits into a top of root_d levels and bottoms of leaf_d levels, leaf_d
// = next power of two >= ceil(d/2) (:240-247).  Layout = [top | full bottoms |
// incomplete bottom]; keys of the top that follow the incomplete bottom in sorted
// order are the roots of the empty bottom slots (:344-380).  Every part is laid
// out recursively with the same rule (:382-413).  The standard van Emde Boas
// layout of the reference's CPU code (cpu/src/veb-cycles.h:33-173) is the same
// recursion with leaf_d = ceil(d/2) unrounded.
#pragma once

#include "tl_common.cuh"

namespace tl {

// ------------------------------------------------------------------ B-tree
struct BtreeGeom {
    uint64_t n = 0, b = 1;
    uint32_t h = 0;       // levels of the perfect top tree
    uint64_t ni = 0;      // keys in the top tree, (b+1)^h - 1
    uint64_t nl = 0;      // keys on the last level
    uint64_t r = 0;       // keys of the partial leaf
    uint64_t l = 0;       // keys of the full leaves
    uint64_t i = 0;       // number of full leaves
    uint64_t lir = 0;     // l + i + r: first sorted rank of the trailing top keys
    uint64_t pw[48];      // (b+1)^k for k <= h + 1 (saturating)
};

TL_HD BtreeGeom make_btree_geom(uint64_t n, uint64_t b) {
    BtreeGeom g;
    g.n = n;
    g.b = b;
    // Exact floor(log_{b+1} n).  The reference's log10(n)/log10(b+1) in double
    // (gpu/src/btree-cycles.cuh:81) agrees wherever its own arithmetic is defined.
    uint32_t h = 0;
    uint64_t p = 1;
    while (n > 0 && p <= n / (b + 1)) {
        p *= (b + 1);
        ++h;
    }
    g.h = h;
    uint64_t q = 1;
    for (uint32_t k = 0; k < 48; ++k) {
        g.pw[k] = q;
        if (q <= UINT64_MAX / (b + 1)) q *= (b + 1); else q = UINT64_MAX;
    }
    g.ni = n ? p - 1 : 0;
    g.nl = n - g.ni;
    g.r = g.nl % b;
    g.l = g.nl - g.r;
    g.i = g.l / b;
    g.lir = g.l + g.i + g.r;
    return g;
}

// Position of top rank c in a perfect B-tree of H levels (levels counted from the
// root).  The level of c is the number of times b+1 divides c+1.
TL_HD uint64_t btree_perfect_pos(const BtreeGeom &g, const FastDiv64 &fd, uint64_t c, uint32_t H) {
    if (g.b == 1) {  // binary tree: the level is the number of trailing zero bits of c+1
        const uint64_t x1 = c + 1;
#ifdef __CUDA_ARCH__
        const uint32_t k = (uint32_t)__ffsll((long long)x1) - 1;
#else
        const uint32_t k = (uint32_t)__builtin_ctzll(x1);
#endif
        return g.pw[H - 1 - k] - 1 + (x1 >> (k + 1));
    }
    uint64_t x = c + 1, q, rem;
    uint32_t k = 0;
    for (;;) {
        fd.divmod(x, q, rem);
        if (rem != 0 || k + 1 >= H) break;
        x = q;
        ++k;
    }
    return g.pw[H - 1 - k] - 1 + q * g.b + rem - 1;
}

// Position of sorted rank s in the B-tree layout.
TL_HD uint64_t btree_pos(const BtreeGeom &g, const FastDiv64 &fd, uint64_t s) {
    uint64_t c;
    if (s < g.l + g.i) {
        uint64_t j, t;
        fd.divmod(s, j, t);
        if (t < g.b) return g.ni + j * g.b + t;
        c = j;
    } else if (s < g.lir) {
        return g.ni + s - g.i;
    } else {
        c = s - g.l - g.r;
    }
    return btree_perfect_pos(g, fd, c, g.h);
}

// Sorted rank of top rank c (inverse of the top-key numbering above).
TL_HD uint64_t btree_top_rank(const BtreeGeom &g, uint64_t c) {
    return c < g.i ? (c + 1) * (g.b + 1) - 1 : c + g.l + g.r;
}

// ------------------------------------------------------------------ mvEB
// Split of a tree of d levels into a top of root_d and bottoms of leaf_d levels:
// root_d = floor((d - 2) / 2) + 1 (cpu/src/veb-cycles.h:118-119,
// gpu/src/mveb-cycles.cuh:240-242), and for the modified layout leaf_d rounded
// up to a power of two (gpu/src/mveb-cycles.cuh:243-246).
TL_HD void veb_split(uint32_t d, bool modified, uint32_t &root_d, uint32_t &leaf_d) {
    root_d = (d - 2) / 2 + 1;
    leaf_d = d - root_d;
    if (modified && (leaf_d & (leaf_d - 1))) {
        uint32_t p = 1;
        while (p < leaf_d) p <<= 1;
        leaf_d = p;
        root_d = d - leaf_d;
    }
}

TL_HD void mveb_split(uint32_t d, uint32_t &root_d, uint32_t &leaf_d) { veb_split(d, true, root_d, leaf_d); }

// Position of sorted rank s in the (modified or standard) vEB layout of n keys.
TL_HD uint64_t veb_pos(uint64_t n, uint64_t s, bool modified) {
    uint64_t pos = 0, nn = n;
    for (;;) {
        if (nn <= 1) return pos;
        uint32_t d = bit_length(nn), rd, ld;
        veb_split(d, modified, rd, ld);
        uint64_t r = low_mask(rd), l = low_mask(ld);
        // full bottom trees: 2^rd of a perfect tree (no division; every level
        // of a perfect layout), else a division, 32-bit when it fits
        uint64_t nf = nn == low_mask(d)          ? r + 1
                      : nn <= 0xFFFFFFFFull ? (uint64_t)((uint32_t)(nn - r) / (uint32_t)l)
                                            : (nn - r) / l;
        uint64_t inc = nn - r - nf * l;
        uint64_t full = nf << ld;  // nf * (l + 1)
        if (s < full) {
            uint64_t i = s >> ld, t = s & l;
            if (t == l) {
                nn = r;
                s = i;
            } else {
                pos += r + i * l;
                nn = l;
                s = t;
            }
        } else if (s < full + inc) {
            pos += r + nf * l;
            s -= full;
            nn = inc;
        } else {
            s = nf + (s - full - inc);
            nn = r;
        }
    }
}

TL_HD uint64_t mveb_pos(uint64_t n, uint64_t s) { return veb_pos(n, s, true); }

// A contiguous source range of the mvEB permutation.  Unit regions (U > 0) hold
// the full bottom trees of one recursion segment: every aligned group of 2^U keys
// is one "unit" (a bottom-level subtree of U levels, 2^U - 1 consecutive ranks
// that land in 2^U - 1 consecutive positions) followed by one separator (a key
// of some tree above it).  Tail regions (U == 0) hold keys that all go through
// the scratch pass.
struct MvebRegion {
    uint64_t src, len;    // source ranks [src, src + len)
    uint64_t dst;         // destination of the segment's top tree
    uint64_t r, l;        // segment's top-tree and bottom-tree sizes
    uint32_t H, U;        // bottom-tree height, unit height (0: tail region)
    uint32_t modified;    // split rule of the layout (1: mvEB, 0: standard vEB)
    uint64_t slot_base;   // first scratch slot of the region
    uint64_t tile_base;   // first tile of the region (tiles ascend with source position)
    uint64_t tile_len;    // keys per tile (a multiple of 2^U)
    uint64_t ntiles;
};

constexpr int kMaxRegions = 40;

struct MvebPlan {
    uint64_t n = 0;
    uint32_t modified = 1;  // 1: mvEB, 0: standard vEB
    int nreg = 0;
    MvebRegion reg[kMaxRegions];
    uint64_t total_slots = 0, total_tiles = 0;
};

// Destination of the first key of unit g (0-based, counted from the start of the
// region) for bottoms of H levels split down to units of U levels: at each split
// of h levels into a top of rt and bottoms of lf levels, every bottom holds
// 2^(lf - U) units, so the unit index picks a bottom with its high bits.
TL_HD uint64_t mveb_unit_dst(const MvebRegion &R, uint64_t g) {
    uint32_t per_bottom_bits = R.H - R.U;
    uint64_t off = R.dst + R.r + (g >> per_bottom_bits) * R.l;
    uint64_t j = g & low_mask(per_bottom_bits);
    uint32_t h = R.H;
    while (h > R.U) {
        uint32_t rt, lf;
        veb_split(h, R.modified != 0, rt, lf);
        const uint32_t jb = lf - R.U;
        off += low_mask(rt) + (j >> jb) * low_mask(lf);
        j &= low_mask(jb);
        h = lf;
    }
    return off;
}

// Height of the units of a bottom of H levels: follow the bottoms of its
// recursion until they have at most unit_max levels.
TL_HD uint32_t veb_unit_levels(uint32_t H, bool modified, uint32_t unit_max) {
    uint32_t h = H;
    while (h > unit_max) {
        uint32_t rt, lf;
        veb_split(h, modified, rt, lf);
        h = lf;
    }
    return h;
}

__host__ inline MvebPlan make_mveb_plan(uint64_t n, uint32_t unit_max_levels, uint64_t tile_keys,
                                       bool modified = true) {
    MvebPlan P;
    P.n = n;
    P.modified = modified ? 1 : 0;
    MvebRegion tails[kMaxRegions];
    int ntails = 0;
    uint64_t src = 0, dst = 0, nn = n;
    while (nn > 0) {
        if (nn == 1) {
            MvebRegion t{};
            t.src = src;
            t.len = 1;
            tails[ntails++] = t;
            break;
        }
        uint32_t d = bit_length(nn), rd, ld;
        veb_split(d, modified, rd, ld);
        uint64_t r = low_mask(rd), l = low_mask(ld);
        // full bottom trees: 2^rd of a perfect tree (no division; every level
        // of a perfect layout), else a division, 32-bit when it fits
        uint64_t nf = nn == low_mask(d)          ? r + 1
                      : nn <= 0xFFFFFFFFull ? (uint64_t)((uint32_t)(nn - r) / (uint32_t)l)
                                            : (nn - r) / l;
        uint64_t inc = nn - r - nf * l;
        uint64_t full = nf << ld;
        MvebRegion u{};
        u.src = src;
        u.len = full < nn ? full : nn;
        u.dst = dst;
        u.r = r;
        u.l = l;
        u.H = ld;
        u.U = veb_unit_levels(ld, modified, unit_max_levels);
        u.modified = P.modified;
        P.reg[P.nreg++] = u;
        uint64_t after = src + full + inc;
        if (full < nn && after < src + nn) {  // roots of the empty bottom slots
            MvebRegion t{};
            t.src = after;
            t.len = src + nn - after;
            tails[ntails++] = t;
        }
        if (inc == 0) break;
        src += full;
        dst += r + nf * l;
        nn = inc;
    }
    for (int k = ntails - 1; k >= 0; --k) P.reg[P.nreg++] = tails[k];
    uint64_t slot = 0, tile = 0;
    for (int k = 0; k < P.nreg; ++k) {
        MvebRegion &R = P.reg[k];
        R.slot_base = slot;
        R.tile_base = tile;
        if (R.U) {
            uint64_t grp = 1ull << R.U;
            R.tile_len = tile_keys < grp ? grp : (tile_keys / grp) * grp;
            slot += (R.len + grp - 1) >> R.U;
        } else {
            R.tile_len = tile_keys;
            slot += R.len;
        }
        R.ntiles = (R.len + R.tile_len - 1) / R.tile_len;
        tile += R.ntiles;
    }
    P.total_slots = slot;
    P.total_tiles = tile;
    return P;
}

}  // namespace tl
