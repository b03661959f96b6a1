// B-tree (and BST, b = 1) streaming permutation: schedules, per-tile index
// helpers (shared by the host replay), and the device bodies of the stream and
// copy passes used by the single-array and the batched kernels.
#pragma once

#include "geometry.cuh"
#include "stream.cuh"

namespace tl {

constexpr int kScatterThreads = 256;     // second-pass kernels (B-tree copy, mvEB scatter)
constexpr uint64_t kCopyChunk = 32768;   // batched mode: keys per copy work item
constexpr int kMaxTopLevels = 36;        // levels of a top tree: a BST of up to 2^37 - 1 keys
constexpr int kMaxTopRuns = 2 * kMaxTopLevels;  // a tile holds at most two groups of top keys

// ---------------------------------------------------------------- B-tree stream
// Two schedules.  Plan R (right to left): the last level's keys go straight to
// their final positions (they move right).  Plan L (left to right), for trees
// whose top tree holds most keys: the top tree's own last level goes straight
// to its final positions (those keys move left) and the last level goes through
// scratch.  A key of the top tree goes straight to its final position p too when
// the tile under p is read before its own tile is: p >= s (its sorted rank) for
// plan R, p <= s for plan L.  On each level of the top tree p - s decreases
// along the level, so those keys form a prefix (plan R) or a suffix (plan L) of
// the level's positions, bounded by bnd[k] (k = 0 is the top tree's last level).
// The other keys go through scratch.  The host picks the plan that moves fewer
// keys through scratch.
//
// Scratch is indexed by final position: slot p holds the key of position p < E
// (the top tree), slot seg1 + (p - ni) the key of position p >= ni (plan L's
// last level).  The second pass is a copy of the scratch ranges (one per level,
// plus the last level under plan L) into place, and the stream pass writes each
// tile's top keys as contiguous runs, one per level.  seg1 is rounded so that
// the copies see the same 16-byte alignment on both sides.
//
// Plan O (ordered) processes the tiles in a host-chosen order, rank[tile] being
// a tile's ticket.  A key of source tile z goes straight to its final position
// p when the tile u under p is z itself or was read before z (rank[u] <
// rank[z]); otherwise it goes to scratch slot p + soff(u).  Only the tiles
// that can receive such keys own scratch (a tile's worth each, in the order of
// the host's list of them), so soff(u) = (slot[u] - u) * tile_keys with slot[u]
// u's index in that list.  rank and slot share one 8-byte entry per tile
// (tab[u]), so a tile's decision and its scratch offset are one load.  The
// order puts each tile before the tile that feeds it most keys, following those
// edges in chains, so that far fewer keys go through scratch than under either
// fixed direction.  Its second pass copies runs of whole scratch tiles with the
// bulk-copy engine and the other scratch keys as host-listed segments
// (btree_fix_kernel).
enum BtreePlan { PLAN_R = 0, PLAN_L = 1, PLAN_O = 2 };

struct BtreeStream {
    BtreeGeom g;
    FastDiv64 fd;         // b + 1
    FastDiv64 fdb;        // b (b >= 2)
    FastDiv32 fd32;       // b + 1, for tile-local offsets
    FastDiv32 fd32b;      // b (unused when b = 1)
    uint64_t tile_keys, ntiles;
    uint32_t tile_shift;  // log2(tile_keys)
    int plan;
    uint64_t i2;          // first position of the top tree's last level, (b+1)^(h-1) - 1
    uint64_t E;           // top-tree scratch slots: [0, E)
    uint64_t seg1;        // plan L: scratch slot of final position ni
    uint64_t nscratch;    // scratch slots
    const uint2 *tab = nullptr;       // plan O: per tile {rank: its ticket, slot: its scratch tile or kNoSlot}
    const uint32_t *order = nullptr;  // plan O: tile of each ticket
    uint64_t bnd[kMaxTopLevels];  // direct-store boundary position of level k
    FastDiv64 pdiv[kMaxTopLevels + 1];  // division by (b+1)^k, k >= 1 (host-built)
};

constexpr uint32_t kNoSlot = 0xFFFFFFFFu;  // tab[u].y of a tile that owns no scratch

// Read-only table loads (the plan-O tables do not change during a launch).
TL_HD uint32_t ld_table(const uint32_t *p) {
#ifdef __CUDA_ARCH__
    return __ldg(p);
#else
    return *p;
#endif
}
TL_HD uint2 ld_entry(const uint2 *p) {
#ifdef __CUDA_ARCH__
    return __ldg(p);
#else
    return *p;
#endif
}

// Records an inconsistent schedule (a scratch store into a tile without scratch).
__device__ __forceinline__ void btree_o_bad(Ctrl *ctrl) { atomicOr(&ctrl->error, 1u << TL_ERROR_UNSUPPORTED); }

// Plan O: tile u's ticket.
TL_HD uint32_t btree_o_rank(const BtreeStream &S, uint64_t u) { return ld_entry(S.tab + u).x; }

// Plan O: may a key of source tile `own` be stored straight into tile u?
TL_HD bool btree_o_direct(const BtreeStream &S, uint64_t own, uint64_t u) {
    return u == own || btree_o_rank(S, u) < btree_o_rank(S, own);
}

// soff of a tile that owns no scratch: any store through it lands far outside
// the scratch, so the kernels check for it (btree_o_bad) before storing.
constexpr int64_t kNoScratch = INT64_MIN;

// The scratch offset of tile u for its entry e = tab[u].
TL_HD int64_t btree_o_soff_of(const BtreeStream &S, uint64_t u, uint2 e) {
    return e.y == kNoSlot ? kNoScratch : ((int64_t)e.y - (int64_t)u) * (int64_t)S.tile_keys;
}

// Plan O: the offset of destination tile u's scratch slots.
TL_HD int64_t btree_o_soff(const BtreeStream &S, uint64_t u) { return btree_o_soff_of(S, u, ld_entry(S.tab + u)); }

// The division table of BtreeStream: pdiv[k] divides by (b+1)^k (k >= 1, while
// that fits 63 bits; larger powers exceed every n and are never used).
struct PowDivs {
    FastDiv64 d[kMaxTopLevels + 1];
};

__host__ inline PowDivs make_pow_divs(uint64_t b) {
    PowDivs P;
    uint64_t q = 1;
    for (int k = 1; k <= kMaxTopLevels; ++k) {
        if (q > (1ull << 62) / (b + 1)) break;
        q *= b + 1;
        P.d[k] = FastDiv64(q);
    }
    return P;
}

TL_HD void btree_set_pow_divs(BtreeStream &S, const PowDivs &P) {
    for (int k = 0; k <= kMaxTopLevels; ++k) S.pdiv[k] = P.d[k];
}

// floor(y / (b+1)^k).
TL_HD uint64_t btree_div_pow(const BtreeStream &S, uint64_t y, uint32_t k) {
    return S.g.b == 1 ? y >> k : k ? S.pdiv[k].div(y) : y;
}

TL_HD uint64_t btree_tile_of_ticket(const BtreeStream &S, uint64_t t) {
    return S.plan == PLAN_R ? S.ntiles - 1 - t : S.plan == PLAN_O ? ld_table(S.order + t) : t;
}

// Source range of tile k (tiles ascend with position).
TL_HD void btree_tile(const BtreeStream &S, uint64_t k, uint64_t &p0, uint64_t &p1) {
    p0 = k << S.tile_shift;
    p1 = p0 + S.tile_keys < S.g.n ? p0 + S.tile_keys : S.g.n;
}

// First position of level k of the top tree (k = 0: its last level) and one
// past its last.
TL_HD uint64_t btree_level_start(const BtreeGeom &g, uint32_t k) { return g.pw[g.h - 1 - k] - 1; }
TL_HD uint64_t btree_level_end(const BtreeGeom &g, uint32_t k) { return g.pw[g.h - k] - 1; }

// Level (k = 0: last) of a top-tree position p < ni.
TL_HD uint32_t btree_level_of(const BtreeGeom &g, uint64_t p) {
    uint32_t L = 0;
    while (L + 1 < g.h && g.pw[L + 1] - 1 <= p) ++L;
    return g.h - 1 - L;
}

// Is the top-tree position p stored directly by the stream pass?
TL_HD bool btree_top_direct(const BtreeStream &S, uint64_t p) {
    const uint64_t bk = S.bnd[btree_level_of(S.g, p)];
    return S.plan == PLAN_R ? p < bk : p >= bk;
}

// Plan R: sorted rank -> destination of a last-level key, extended monotonically
// over the separators in between; bounds the destinations of a tile.
TL_HD uint64_t btree_leaf_dest_bound(const BtreeStream &S, uint64_t s) {
    return s < S.g.l + S.g.i ? S.g.ni + s - S.fd.div(s) : S.g.ni + s - S.g.i;
}

// Plan L: sorted rank s >= lir (top rank c) -> destination of a key of the top
// tree's last level, extended monotonically over the upper keys.
TL_HD uint64_t btree_top_last_dest_bound(const BtreeStream &S, uint64_t s) {
    const uint64_t c = s - S.g.l - S.g.r;
    return S.i2 + c - S.fd.div(c + 1);
}

// Tiles (other than k) whose source lies under the destinations of the tile's
// bulk keys (plan R: its last-level keys; plan L: its keys of the top tree's
// last level): right of the tile for plan R, left of it for plan L, i.e.
// always tiles with earlier tickets.  False if there are none.  Plan O: every
// tile under the destinations of the tile's bulk keys (last-level keys, or on a
// tail tile its keys of the top tree's last level); the caller waits only for
// those that take direct stores (btree_o_direct).
TL_HD bool btree_tile_wait(const BtreeStream &S, uint64_t p0, uint64_t p1, uint64_t &k_lo, uint64_t &k_hi) {
    const BtreeGeom &g = S.g;
    if (S.plan == PLAN_O && p0 >= g.lir && g.lir < g.n) {  // tail tile: its top-last-level keys are bulk
        const uint64_t d0 = btree_top_last_dest_bound(S, p0), d1 = btree_top_last_dest_bound(S, p1 - 1) + 1;
        k_lo = d0 >> S.tile_shift;
        k_hi = (d1 - 1) >> S.tile_shift;
        return true;
    }
    if (S.plan != PLAN_L) {
        if (p0 >= g.lir) return false;
        uint64_t d0 = btree_leaf_dest_bound(S, p0);
        uint64_t d1 = btree_leaf_dest_bound(S, (p1 < g.lir ? p1 : g.lir) - 1) + 1;
        if (d1 > g.n) d1 = g.n;  // a trailing separator bounds past the last leaf key
        uint64_t lo = S.plan == PLAN_O ? d0 : d0 > p1 ? d0 : p1;
        if (lo >= d1) return false;
        k_lo = lo >> S.tile_shift;
        k_hi = (d1 - 1) >> S.tile_shift;
        return true;
    }
    if (p1 <= g.lir) return false;
    uint64_t d0 = btree_top_last_dest_bound(S, p0 > g.lir ? p0 : g.lir);
    uint64_t d1 = btree_top_last_dest_bound(S, p1 - 1) + 1;
    uint64_t hi = d1 < p0 ? d1 : p0;
    if (d0 >= hi) return false;
    k_lo = d0 >> S.tile_shift;
    k_hi = (hi - 1) >> S.tile_shift;
    return true;
}

// Scratch slot of a final position that goes through scratch.
TL_HD uint64_t btree_scratch_slot(const BtreeStream &S, uint64_t p) {
    if (S.plan == PLAN_O) return p + (uint64_t)btree_o_soff(S, p >> S.tile_shift);
    return p < S.g.ni ? p : p - S.g.ni + S.seg1;
}

// Where sorted rank x goes in the stream pass: true -> A[idx] (final position),
// false -> scratch[idx].
TL_HD bool btree_place(const BtreeStream &S, uint64_t x, uint64_t &idx) {
    const uint64_t p = btree_pos(S.g, S.fd, x);
    const bool direct = S.plan == PLAN_O ? btree_o_direct(S, x >> S.tile_shift, p >> S.tile_shift)
                        : p >= S.g.ni    ? S.plan == PLAN_R
                                         : btree_top_direct(S, p);
    idx = direct ? p : btree_scratch_slot(S, p);
    return direct;
}

// Sorted rank of the key at layout position p (the inverse of btree_pos).  On
// level k of the top tree the t-th position holds x = t + 1 + floor(t / b),
// i.e. top rank c = x (b+1)^k - 1; on the last level the j-th position holds
// full-leaf key j + floor(j / b) or, past them, partial-leaf key j + i.
TL_HD uint64_t btree_src_rank(const BtreeStream &S, uint64_t p) {
    const BtreeGeom &g = S.g;
    if (p >= g.ni) {
        const uint64_t j = p - g.ni;
        if (j >= g.l) return j + g.i;
        return j + (g.b == 1 ? j : S.fdb.div(j));
    }
    const uint32_t k = btree_level_of(g, p);
    const uint64_t t = p - btree_level_start(g, k);
    const uint64_t q = g.b == 1 ? t : S.fdb.div(t);
    const uint64_t x = t + 1 + q;
    return btree_top_rank(g, x * g.pw[k] - 1);
}

constexpr uint32_t kLastLevel = 0xFFFFFFFFu;  // level index of the B-tree's last level

// First position of level lv (kLastLevel, or k < h of the top tree) whose key
// has sorted rank >= sr, or the level's end.  Sorted rank grows with position
// along a level, so the positions of one source tile form a run.
TL_HD uint64_t btree_first_pos(const BtreeStream &S, uint32_t lv, uint64_t sr) {
    const BtreeGeom &g = S.g;
    if (lv == kLastLevel) {
        uint64_t j;
        if (sr >= g.l + g.i) {
            j = sr - g.i;
        } else {
            uint64_t q, t;
            S.fd.divmod(sr, q, t);
            j = q * g.b + (t < g.b ? t : g.b);  // a separator (t = b) passes to the next leaf
        }
        return g.ni + (j < g.nl ? j : g.nl);
    }
    const uint64_t ls = btree_level_start(g, lv), le = btree_level_end(g, lv);
    // smallest top rank c with btree_top_rank(c) >= sr: (c+1)(b+1) - 1 >= sr
    // among the separators, c + l + r >= sr after them
    uint64_t c = S.fd.div(sr + g.b + 1) - 1;
    if (c >= g.i) {
        const uint64_t lr = g.l + g.r;
        c = sr > lr + g.i ? sr - lr : g.i;
    }
    // smallest x, not a multiple of b+1, with x (b+1)^lv - 1 >= c
    const uint64_t x0 = btree_div_pow(S, c + g.pw[lv], lv);
    uint64_t q, rem;
    S.fd.divmod(x0, q, rem);
    const uint64_t t = q * g.b + (rem ? rem : 1) - 1;
    return ls + t < le ? ls + t : le;
}

// Plan O on top of a geometry, with scratch for `scratch_tiles` destination tiles.
TL_HD void btree_set_ordered(BtreeStream &S, const uint2 *tab, const uint32_t *order, uint64_t scratch_tiles) {
    S.plan = PLAN_O;
    S.tab = tab;
    S.order = order;
    S.E = 0;
    S.seg1 = S.g.ni;
    S.nscratch = scratch_tiles * S.tile_keys;
}

// Is sorted rank x a key of the top tree?
TL_HD bool btree_is_top(const BtreeStream &S, uint64_t x) {
    const BtreeGeom &g = S.g;
    if (x < g.l + g.i) return x - S.fd.div(x) * (g.b + 1) == g.b;
    return x >= g.lir;
}

// Position of the level-k key with multiplier x (top rank c = x (b+1)^k - 1)
// and its sorted rank; for a multiple x of b+1 the position is that of the
// previous non-multiple, which keeps p non-decreasing in x.
TL_HD void btree_level_key(const BtreeStream &S, uint32_t k, uint64_t x, uint64_t &p, uint64_t &s) {
    p = btree_level_start(S.g, k) + (x - S.fd.div(x)) - 1;
    s = btree_top_rank(S.g, x * S.g.pw[k] - 1);
}

// bnd[k] for every level: along a level p - s strictly decreases with x, so a
// binary search over x finds where the direct condition flips.  Level k holds
// x in [1, xmax], xmax = (b+1)^(h-k) - 1; the t-index of the last non-multiple
// <= x is T(x) - 1, T(x) = x - floor(x / (b+1)).
TL_HD void btree_direct_bounds(BtreeStream &S) {
    const BtreeGeom &g = S.g;
    for (uint32_t k = 0; k < g.h; ++k) {
        const uint64_t ls = btree_level_start(g, k), xmax = g.pw[g.h - k] - 1;
        uint64_t p, s;
        if (S.plan == PLAN_R) {  // largest x with p >= s
            btree_level_key(S, k, 1, p, s);
            if (p < s) {
                S.bnd[k] = ls;
                continue;
            }
            uint64_t lo = 1, hi = xmax;
            while (lo < hi) {
                const uint64_t mid = lo + (hi - lo + 1) / 2;
                btree_level_key(S, k, mid, p, s);
                if (p >= s) lo = mid; else hi = mid - 1;
            }
            S.bnd[k] = ls + lo - S.fd.div(lo);
        } else {  // smallest x with p <= s
            btree_level_key(S, k, xmax, p, s);
            if (p > s) {
                S.bnd[k] = btree_level_end(g, k);
                continue;
            }
            uint64_t lo = 1, hi = xmax;
            while (lo < hi) {
                const uint64_t mid = lo + (hi - lo) / 2;
                btree_level_key(S, k, mid, p, s);
                if (p <= s) hi = mid; else lo = mid + 1;
            }
            S.bnd[k] = ls + (lo - 1) - S.fd.div(lo - 1);
        }
    }
}

// Keys a plan moves through scratch (its second pass reads and writes each once).
TL_HD uint64_t btree_scratch_traffic(const BtreeStream &S) {
    const BtreeGeom &g = S.g;
    uint64_t keys = S.plan == PLAN_L ? g.nl : 0;
    for (uint32_t k = 0; k < g.h; ++k) {
        const uint64_t ls = btree_level_start(g, k), le = btree_level_end(g, k), bk = S.bnd[k];
        keys += S.plan == PLAN_R ? le - (bk > ls ? bk : ls) : (bk < le ? bk : le) - ls;
    }
    return keys;
}

TL_HD void btree_choose_plan(BtreeStream &S, uint32_t key_bytes) {
    const BtreeGeom &g = S.g;
    S.plan = PLAN_R;
    S.i2 = g.h >= 1 ? g.pw[g.h - 1] - 1 : 0;
    S.E = g.ni;
    S.seg1 = g.ni;
    S.nscratch = g.ni;
    if (g.h < 1) return;
    btree_direct_bounds(S);
    // Plan L needs every key of the top tree's last level beyond the separators
    // (top ranks c >= i) to move left: i2 <= l + r + floor((c+1)/(b+1)) at c = i.
    if (g.lir >= g.n) return;
    if (S.i2 > g.l + g.r + (g.i + 1) / (g.b + 1)) return;
    BtreeStream L = S;
    L.plan = PLAN_L;
    btree_direct_bounds(L);
    if (btree_scratch_traffic(L) >= btree_scratch_traffic(S)) return;
    // the top-tree scratch ends where level 0's direct suffix starts (upper
    // levels lie below i2 <= bnd[0])
    const uint64_t vec = 16 / key_bytes;
    L.E = L.bnd[0];
    L.seg1 = L.E + (g.ni - L.E) % vec;  // seg1 == ni (mod 16 bytes / key)
    L.nscratch = L.seg1 + g.nl;
    S = L;
}

// Is scratch slot `slot` written by the stream pass?
TL_HD bool btree_slot_used(const BtreeStream &S, uint64_t slot) {
    if (slot < S.E) return slot < S.g.ni && !btree_top_direct(S, slot);
    return S.plan == PLAN_L && slot >= S.seg1 && slot < S.seg1 + S.g.nl;
}

// Per-tile fast paths.  Inside most tiles the keys that are not keys of the
// top tree ("bulk" keys) follow one rule: with v = r0 + o (o = x - p0, r0 a
// remainder fixed per tile) and ql = v / (b+1), rem = v - ql (b+1), the key goes
// to tgt[dbase + v - ql] (tgt = A or scratch) unless rem == skip (a top key).
// Top keys come in at most two groups of consecutive top ranks c, c + 1 in
// [y_lo, y_hi], the key of c sitting at tile offset (c + 1) f - gneg: the
// separators between full leaves (f = b+1) and the trailing top keys (f = 1).
// They are stored as one contiguous run per level (levels >= kmin).
// kind 1: bulk fast path + top runs; kind 2: top runs only; kind 0: the tile
// straddles a region boundary, its bulk keys take btree_place one by one.
//
// Derivations.  Plan R, x < l + i: x = j (b+1) + t, a leaf key (t < b) lands at
// ni + j b + t = ni + q0 b + v - ql, a separator (t = b) is top rank j, at
// offset (j + 1)(b+1) - 1 - p0.  Plan L, x >= lir: c = x - l - r, c + 1 =
// q (b+1) + rem; rem != 0 puts it on the top tree's last level at
// i2 + (c + 1) - q - 1 = i2 + q0 b - 1 + v - ql (always direct under plan L),
// rem == 0 on a level above.
struct TopGroup {
    uint64_t y_lo, y_hi, f, gneg;
    uint32_t kmin;
};

// kind 3 (plan O, full leaves): kind 1 with targets per destination tile: bulk
// indices below dsplit go to A when to_A, else to scratch at index + slo; the
// others to A when hi_A, else to scratch at index + shi.
struct Regime {
    int kind;
    bool to_A, hi_A;
    uint32_t r0, skip;
    uint64_t dbase, dsplit;
    int64_t slo, shi;
};

TL_HD TopGroup btree_sep_group(const BtreeStream &S, uint64_t p0, uint64_t end) {
    TopGroup G;
    G.y_lo = S.fd.div(p0 + 1 + S.g.b);  // ceil((p0 + 1) / (b+1))
    G.y_hi = S.fd.div(end);
    G.f = S.g.b + 1;
    G.gneg = p0 + 1;
    G.kmin = 0;
    return G;
}

TL_HD TopGroup btree_tail_group(const BtreeStream &S, uint64_t p0, uint64_t start, uint64_t p1, uint32_t kmin) {
    const BtreeGeom &g = S.g;
    TopGroup G;
    G.y_lo = start - g.l - g.r + 1;
    G.y_hi = p1 - g.l - g.r;
    G.f = 1;
    G.gneg = p0 + 1 - g.l - g.r;
    G.kmin = kmin;
    return G;
}

// Plan O: a kind-1 regime's bulk indices start at that of its first non-skip
// offset and span fewer than tile_keys positions, i.e. at most two destination
// tiles; kind 3 splits them there.
TL_HD void btree_regime_split(const BtreeStream &S, uint64_t p0, Regime &R) {
    const uint32_t d = (uint32_t)S.g.b + 1;
    const uint32_t v0 = R.r0 == R.skip ? R.r0 + 1 : R.r0;
    const uint64_t own = p0 >> S.tile_shift, u0 = (R.dbase + v0 - v0 / d) >> S.tile_shift;
    R.kind = 3;
    R.dsplit = (u0 + 1) << S.tile_shift;
    const bool two = u0 + 1 < S.ntiles;
    const uint32_t ro = btree_o_rank(S, own);
    const uint2 e0 = ld_entry(S.tab + u0), e1 = two ? ld_entry(S.tab + u0 + 1) : make_uint2(0, kNoSlot);
    R.to_A = u0 == own || e0.x < ro;
    R.hi_A = !two || u0 + 1 == own || e1.x < ro;
    R.slo = R.to_A ? 0 : btree_o_soff_of(S, u0, e0);
    R.shi = R.hi_A ? 0 : btree_o_soff_of(S, u0 + 1, e1);
}

TL_HD Regime btree_stream_regime(const BtreeStream &S, uint64_t p0, uint64_t p1) {
    const BtreeGeom &g = S.g;
    Regime R{};
    if (g.h == 0) return R;  // no top tree: kind 0
    uint64_t q0, r0;
    if (p1 <= g.l + g.i) {  // full leaves and their separators
        S.fd.divmod(p0, q0, r0);
        R.kind = 1;
        R.r0 = (uint32_t)r0;
        R.skip = (uint32_t)g.b;
        R.to_A = S.plan != PLAN_L;
        R.dbase = R.to_A ? g.ni + q0 * g.b : S.seg1 + q0 * g.b;
        if (S.plan == PLAN_O) btree_regime_split(S, p0, R);
    } else if (p0 >= g.lir) {  // trailing top keys
        if (S.plan == PLAN_R) {
            R.kind = 2;
        } else {
            S.fd.divmod(p0 - g.l - g.r + 1, q0, r0);
            R.kind = 1;
            R.r0 = (uint32_t)r0;
            R.skip = 0;
            R.to_A = true;
            R.dbase = S.i2 + q0 * g.b - 1;
            if (S.plan == PLAN_O) btree_regime_split(S, p0, R);
        }
    }
    return R;
}

// The tile's groups of top keys (levels kmin.. of each); returns their number.
// Under plans L and O a tail tile's keys of the top tree's last level are bulk keys.
TL_HD int btree_stream_groups(const BtreeStream &S, uint64_t p0, uint64_t p1, TopGroup &G0, TopGroup &G1) {
    const BtreeGeom &g = S.g;
    if (g.h == 0) return 0;
    const uint64_t li = g.l + g.i;
    if (p1 <= li) {
        G0 = btree_sep_group(S, p0, p1);
        return 1;
    }
    if (p0 >= g.lir) {
        G0 = btree_tail_group(S, p0, p0, p1, S.plan == PLAN_R ? 0 : 1);
        return 1;
    }
    int ng = 0;
    if (p0 < li) {
        G0 = btree_sep_group(S, p0, p1 < li ? p1 : li);
        ++ng;
    }
    if (p1 > g.lir) {
        (ng ? G1 : G0) = btree_tail_group(S, p0, p0 > g.lir ? p0 : g.lir, p1, 0);
        ++ng;
    }
    return ng;
}

// Bulk-key form of btree_place for offset o of a kind-1 tile: true with the
// target index, or false for a top key.
TL_HD bool btree_regime_bulk(const BtreeStream &S, const Regime &R, uint32_t o, uint64_t &idx) {
    const uint32_t v = R.r0 + o;
    const uint32_t ql = S.fd32.div(v);
    if (v - ql * S.fd32.d == R.skip) return false;
    idx = R.dbase + (v - ql);
    return true;
}

// Kind 3: every part of the bulk range that goes to scratch has scratch.
TL_HD bool btree_regime_ok(const BtreeStream &S, const Regime &R, uint32_t cnt) {
    const uint32_t d = S.fd32.d;
    uint32_t v0 = R.r0, v1 = R.r0 + cnt - 1;  // first and last bulk offsets (+ r0)
    if (v0 % d == R.skip) ++v0;
    if (v1 % d == R.skip) --v1;
    if (cnt == 0 || v0 > v1) return true;
    const uint64_t i0 = R.dbase + v0 - v0 / d, i1 = R.dbase + v1 - v1 / d;
    if (i0 < R.dsplit && !R.to_A && R.slo == kNoScratch) return false;
    if (i1 >= R.dsplit && !R.hi_A && R.shi == kNoScratch) return false;
    return true;
}

// One level's run of top keys inside a tile.  Level k holds the top ranks with
// c + 1 = x (b+1)^k, x not a multiple of b+1; the t-th such x (t counted from 0
// over the whole level) is x = t + 1 + floor(t / b) and lands at
// btree_level_start(k) + t.  Element e of a run (t = t0 + e) has
// x = xb + e + floor((rb + e) / b), xb the run's first x and rb + 1 its
// remainder mod b+1, and sits at tile offset x * mult - gneg (mult = (b+1)^k f),
// i.e. off0 + (e + floor((rb + e) / b)) * mult with off0 = xb * mult - gneg.
// Offsets are below the tile size, so they are computed modulo 2^32.  Elements
// [0, nlo) of the run go to A when bit 0 of `direct` is set, the rest when bit
// 1 is; otherwise to scratch, at the position (plans R, L) or at the position +
// slo / shi (plan O).  Under plan R nlo splits at bnd[k] with direct = 1, under
// plan L with direct = 2; under plan O nlo is where the run crosses into the
// next destination tile.
struct TopRun {
    uint64_t dest0;
    int64_t slo, shi;
    uint32_t off0, mult, rb, cnt, nlo, direct;
};

// The run of level k of a group of top keys (cnt = 0 when empty).  With hi_k =
// floor(y_hi / (b+1)^k) and lo_k = floor((y_lo - 1) / (b+1)^k), level k holds
// the non-multiples of b+1 in (lo_k, hi_k]: t0 = lo_k - lo_{k+1} of them lie at
// or below lo_k, and (hi_k - hi_{k+1}) - t0 in the range (hi_{k+1} =
// floor(hi_k / (b+1))).  A tile's runs occupy slots s = group * kMaxTopLevels +
// level; slots of levels below kmin or above the tree are empty.
TL_HD TopRun btree_group_run(const BtreeStream &S, const TopGroup &G, uint32_t k, uint64_t own) {
    const BtreeGeom &g = S.g;
    TopRun run{};
    if (k < G.kmin || k >= g.h || G.y_lo > G.y_hi) return run;
    const uint64_t hi = btree_div_pow(S, G.y_hi, k), lo = btree_div_pow(S, G.y_lo - 1, k);
    if (hi <= lo) return run;
    const uint64_t d = g.b + 1;
    const uint64_t hi1 = S.fd.div(hi), lo1 = S.fd.div(lo);
    const uint64_t t0 = lo - lo1, t1 = hi - hi1;
    if (t1 <= t0) return run;
    run.cnt = (uint32_t)(t1 - t0);
    uint64_t rem = lo - lo1 * d + 1;  // the first non-multiple of b+1 above lo, and its remainder
    uint64_t xb = lo + 1;
    if (rem == d) {
        xb = lo + 2;
        rem = 1;
    }
    run.rb = (uint32_t)(rem - 1);
    run.dest0 = btree_level_start(g, k) + t0;
    const uint64_t mult = g.pw[k] * G.f;
    run.mult = (uint32_t)mult;
    run.off0 = (uint32_t)(xb * mult - G.gneg);
    if (S.plan == PLAN_O) {  // a run spans fewer than tile_keys positions: at most two tiles
        const uint64_t u0 = run.dest0 >> S.tile_shift, split = (u0 + 1) << S.tile_shift;
        run.nlo = split - run.dest0 < run.cnt ? (uint32_t)(split - run.dest0) : run.cnt;
        const bool two = run.nlo < run.cnt;
        const uint32_t ro = btree_o_rank(S, own);
        const uint2 e0 = ld_entry(S.tab + u0), e1 = two ? ld_entry(S.tab + u0 + 1) : make_uint2(0, kNoSlot);
        const bool d0 = u0 == own || e0.x < ro, d1 = two && (u0 + 1 == own || e1.x < ro);
        run.direct = (d0 ? 1u : 0u) | (d1 ? 2u : 0u);
        if (!d0) run.slo = btree_o_soff_of(S, u0, e0);
        if (two && !d1) run.shi = btree_o_soff_of(S, u0 + 1, e1);
        return run;
    }
    const uint64_t bk = S.bnd[k];
    run.nlo = bk <= run.dest0 ? 0 : (bk - run.dest0 < run.cnt ? (uint32_t)(bk - run.dest0) : run.cnt);
    run.direct = S.plan == PLAN_R ? 1u : 2u;
    return run;
}


// Tile offset of element e of a run.
template <class Run>
TL_HD uint32_t btree_top_item_off(const BtreeStream &S, const Run &run, uint32_t e) {
    const uint32_t qe = S.g.b == 1 ? e : S.fd32b.div(run.rb + e);  // b = 1: rb = 0
    return run.off0 + (e + qe) * run.mult;
}

// Does element e of a run go straight to A?
TL_HD bool btree_run_direct(const BtreeStream &S, const TopRun &run, uint32_t e) {
    return (run.direct >> (e < run.nlo ? 0 : 1)) & 1u;
}

// Tiles under the direct part of a run (all with earlier tickets, or the tile
// itself); false when the run has no direct part.
TL_HD bool btree_run_wait(const BtreeStream &S, const TopRun &run, uint64_t &k_lo, uint64_t &k_hi) {
    const uint32_t e0 = (run.direct & 1u) ? 0 : run.nlo, e1 = (run.direct & 2u) ? run.cnt : run.nlo;
    if (e0 >= e1) return false;
    k_lo = (run.dest0 + e0) >> S.tile_shift;
    k_hi = (run.dest0 + e1 - 1) >> S.tile_shift;
    return true;
}

// What the block's store loop needs of a run: for element e, the key at tile
// offset btree_top_item_off goes to (e < nlo ? blo : bhi)[e], the two bases
// being the run's first destination in A or in the scratch.
struct StoreRun {
    uint64_t blo, bhi;
    uint32_t off0, mult, rb, nlo;
};

// Shared-memory workspace of btree_stream_tile.
struct TileShared {
    StoreRun runs[kMaxTopRuns];
    uint32_t cum[kMaxTopRuns + 1];
    uint32_t nslots;
    int ok0, ok1;  // warp 0's and warps 1..'s waits all ended (and no schedule error)
    Regime reg;
};

// Warp 0's part of btree_stream_tile: the tile's runs (one lane per slot, a
// slot per level of each group of top keys, with their plan-O table lookups),
// their prefix sums and store bases, and the waits for the tiles under their
// direct parts.  Kept out of line so that its 64-bit state does not crowd the
// registers of the tile loops.
static __device__ __noinline__ void btree_tile_runs_warp(const BtreeStream &S, uint64_t p0, uint64_t p1,
                                                         uintptr_t ab, uintptr_t sb, uint32_t kb,
                                                         unsigned int *flags, Ctrl *ctrl, const WaitCfg &wc,
                                                         TileShared &ts) {
    const uint32_t lane = threadIdx.x;
    const uint64_t own = p0 >> S.tile_shift;
    TopGroup G0{}, G1{};
    const int ng = btree_stream_groups(S, p0, p1, G0, G1);
    const uint32_t h = S.g.h, nslots = (uint32_t)ng * h;  // slot = group * h + level
    uint32_t carry = 0;
    for (uint32_t s0 = 0; s0 < nslots; s0 += 32) {
        const uint32_t sl = s0 + lane;
        TopRun run{};
        if (sl < nslots) run = btree_group_run(S, sl < h ? G0 : G1, sl < h ? sl : sl - h, own);
        uint32_t incl = run.cnt;
#pragma unroll
        for (int dd = 1; dd < 32; dd <<= 1) {
            const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, dd);
            if (lane >= (uint32_t)dd) incl += y;
        }
        if (S.plan == PLAN_O && run.cnt &&
            ((run.nlo && !(run.direct & 1u) && run.slo == kNoScratch) ||
             (run.nlo < run.cnt && !(run.direct & 2u) && run.shi == kNoScratch))) {
            btree_o_bad(ctrl);
            ts.ok0 = 0;
        }
        if (sl < nslots) {
            StoreRun sr;
            const uintptr_t d0 = (uintptr_t)run.dest0 * kb;
            sr.blo = (run.direct & 1u) ? ab + d0 : sb + d0 + (uintptr_t)run.slo * kb;
            sr.bhi = (run.direct & 2u) ? ab + d0 : sb + d0 + (uintptr_t)run.shi * kb;
            sr.off0 = run.off0;
            sr.mult = run.mult;
            sr.rb = run.rb;
            sr.nlo = run.nlo;
            ts.runs[sl] = sr;
            ts.cum[sl] = carry + incl - run.cnt;
        }
        carry += __shfl_sync(0xFFFFFFFFu, incl, 31);
        uint64_t r_lo, r_hi;
        if (run.cnt && btree_run_wait(S, run, r_lo, r_hi))
            for (uint64_t f = r_lo; f <= r_hi; ++f)
                if (!wait_flag(&flags[f], wc.wait_value, ctrl, wc)) ts.ok0 = 0;
    }
    if (lane == 0) {
        ts.cum[nslots] = carry;
        ts.nslots = nslots;
    }
}

// Named barrier among the threads of warps 1.. of the block.
__device__ __forceinline__ void bar_sync_tail() {
    asm volatile("bar.sync 1, %0;" ::"r"(blockDim.x - 32) : "memory");
}

// Stream pass for tile k of one array (block-wide).  False if a bounded wait
// expired (the tile's stores were skipped and the error is recorded).  Warps
// 1.. load the tile, publish it and store its bulk keys (after waiting for the
// tiles under them); meanwhile warp 0 computes the tile's runs of top keys (one
// lane per level, with their table lookups) and waits for the tiles under
// their direct parts, so that its work stays off the load's path.  Then the
// whole block stores the top keys.  Every wait is on a tile with an earlier
// ticket, and the publish does not depend on warp 0.  kRunRegs keeps the
// current store run in registers across the top-key loop instead of reading it
// from shared memory for every key (the BST instance: many short runs per
// tile; measured +3 % there, but not for b = 16, whose kernel keeps the
// shared-memory reads and its lower register count).
template <typename K, bool kRunRegs = false>
__device__ __forceinline__ bool btree_stream_tile(const BtreeStream &S, K *__restrict__ A, K *__restrict__ scr,
                                                  unsigned int *flags, Ctrl *ctrl, const WaitCfg &wc, uint64_t k,
                                                  K *sm, TileShared &ts) {
    uint64_t p0, p1;
    btree_tile(S, k, p0, p1);
    const uint64_t base = tile_base(A, p0);
    const uint32_t cnt = (uint32_t)(p1 - p0);
    const K *tile = sm + (p0 - base);
    if (threadIdx.x < 32) {
        if (threadIdx.x == 0) ts.ok0 = 1;  // the previous tile's readers are past the ticket barrier
        __syncwarp();
        btree_tile_runs_warp(S, p0, p1, reinterpret_cast<uintptr_t>(A), reinterpret_cast<uintptr_t>(scr),
                             (uint32_t)sizeof(K), flags, ctrl, wc, ts);
    } else {
        const uint32_t tb = threadIdx.x - 32, nb = blockDim.x - 32;
        if (tb == 0) {
            ts.ok1 = 1;
            ts.reg = btree_stream_regime(S, p0, p1);
        }
        load_tile_issue(A, p0, p1, sm, tb, nb);
        load_tile_wait();
        bar_sync_tail();  // the tile is in shared memory
        if (tb == 0) st_relaxed(&flags[k], wc.flag_value);  // published: every copy has landed
        uint64_t w_lo, w_hi;
        if (btree_tile_wait(S, p0, p1, w_lo, w_hi))
            for (uint64_t f = w_lo + tb; f <= w_hi; f += nb) {
                if (S.plan == PLAN_O && !btree_o_direct(S, k, f)) continue;  // its keys go to scratch
                if (!wait_flag(&flags[f], wc.wait_value, ctrl, wc)) ts.ok1 = 0;
            }
        bar_sync_tail();
        if (ts.ok1) {
            const Regime &R = ts.reg;  // fields read from shared memory where used
            if (R.kind == 0) {
                for (uint64_t x = p0 + tb; x < p1; x += nb) {
                    if (btree_is_top(S, x)) continue;
                    uint64_t idx;
                    const K key = sm[x - base];
                    if (btree_place(S, x, idx))
                        A[idx] = key;
                    else if (idx < S.nscratch)
                        scr[idx] = key;
                    else
                        btree_o_bad(ctrl);
                }
            } else if (R.kind == 1) {
                // the loops keep the regime in registers (stores through K * could alias it)
                K *tgt = (R.to_A ? A : scr) + R.dbase;
                const uint32_t d = S.fd32.d, r0 = R.r0, skip = R.skip;
#pragma unroll 4
                for (uint32_t o = tb; o < cnt; o += nb) {
                    const uint32_t v = r0 + o;
                    const uint32_t ql = S.fd32.div(v);
                    if (v - ql * d != skip) tgt[v - ql] = tile[o];
                }
            } else if (R.kind == 3 && !btree_regime_ok(S, R, cnt)) {
                if (tb == 0) btree_o_bad(ctrl);
            } else if (R.kind == 3) {
                K *tlo = (R.to_A ? A : scr + R.slo) + R.dbase, *thi = (R.hi_A ? A : scr + R.shi) + R.dbase;
                const uint32_t d = S.fd32.d, r0 = R.r0, skip = R.skip;
                const uint32_t split = (uint32_t)(R.dsplit - R.dbase);  // below tile_keys + b
#pragma unroll 4
                for (uint32_t o = tb; o < cnt; o += nb) {
                    const uint32_t v = r0 + o;
                    const uint32_t ql = S.fd32.div(v);
                    const uint32_t j = v - ql;
                    if (v - ql * d != skip) (j < split ? tlo : thi)[j] = tile[o];
                }
            }
        }
    }
    __syncthreads();
    if (!ts.ok0 || !ts.ok1) return false;
    // top keys, level by level: consecutive threads store consecutive positions
    const uint32_t total = ts.cum[ts.nslots];
    uint32_t r = 0;  // the run of gi only moves forward as gi grows
    if constexpr (kRunRegs) {
        uint32_t c0 = ts.cum[0], c1 = ts.cum[1];
        StoreRun run = ts.runs[0];
        for (uint32_t gi = threadIdx.x; gi < total; gi += blockDim.x) {
            if (gi >= c1) {
                do {
                    ++r;
                } while (gi >= ts.cum[r + 1]);
                c0 = ts.cum[r];
                c1 = ts.cum[r + 1];
                run = ts.runs[r];
            }
            const uint32_t e = gi - c0;
            K *dst = reinterpret_cast<K *>(e < run.nlo ? run.blo : run.bhi);
            dst[e] = tile[btree_top_item_off(S, run, e)];
        }
    } else {
        for (uint32_t gi = threadIdx.x; gi < total; gi += blockDim.x) {
            while (gi >= ts.cum[r + 1]) ++r;
            const StoreRun run = ts.runs[r];
            const uint32_t e = gi - ts.cum[r];
            K *dst = reinterpret_cast<K *>(e < run.nlo ? run.blo : run.bhi);
            dst[e] = tile[btree_top_item_off(S, run, e)];
        }
    }
    return true;
}

// ---------------------------------------------------------------- plan O second pass
// Destination tile u's positions split into one piece per level; along a piece
// the source tiles z0..z1 of its keys come in runs of consecutive positions
// (btree_first_pos).  The run of source tile z went to scratch iff z != u and
// rank[z] < rank[u] (z was processed before u was read).

// The piece of tile u's positions that starts at position a: its level and end.
TL_HD void btree_fix_piece(const BtreeStream &S, uint64_t a, uint64_t P1, uint32_t &lv, uint64_t &e) {
    const BtreeGeom &g = S.g;
    if (a >= g.ni) {
        lv = kLastLevel;
        e = P1;
        return;
    }
    lv = btree_level_of(g, a);
    const uint64_t le = btree_level_end(g, lv);
    e = le < P1 ? le : P1;
}

// Positions [pa, pe) of source tile z within the piece [a, e) of level lv whose
// source tiles run from z0 to z1.
TL_HD void btree_fix_run(const BtreeStream &S, uint32_t lv, uint64_t a, uint64_t e, uint64_t z0, uint64_t z1,
                         uint64_t z, uint64_t &pa, uint64_t &pe) {
    pa = z == z0 ? a : btree_first_pos(S, lv, z << S.tile_shift);
    pe = z == z1 ? e : btree_first_pos(S, lv, (z + 1) << S.tile_shift);
    if (pa < a) pa = a;
    if (pe > e) pe = e;
    if (pe < pa) pe = pa;
}

// Sorted rank of position p on level lv (kLastLevel or a top level): the
// inverse of btree_pos without the level search.
TL_HD uint64_t btree_src_rank_at(const BtreeStream &S, uint32_t lv, uint64_t p) {
    const BtreeGeom &g = S.g;
    if (lv == kLastLevel) {
        const uint64_t j = p - g.ni;
        return j >= g.l ? j + g.i : j + (g.b == 1 ? j : S.fdb.div(j));
    }
    const uint64_t t = p - btree_level_start(g, lv);
    const uint64_t x = t + 1 + (g.b == 1 ? t : S.fdb.div(t));
    return btree_top_rank(g, x * g.pw[lv] - 1);
}

// Host form (replay, scratch lists and counts): calls visit(pa, len) for each
// scratch run of tile u (positions; u's slots are at position + soff[u]) until
// visit returns false.  Same two cases as the device form below: a piece with
// few source tiles by source runs, any other position by position.
template <class Visit>
__host__ void btree_fix_tile_host(const BtreeStream &S, uint64_t u, Visit &&visit);

// The device side of the fix pass copies host-listed segments (each made of
// these runs) with warp_copy_keys.  Host enumeration: a piece with few source
// tiles (below kFixDense) run by run, any other position by position.
constexpr int kFixUnr = 8;
constexpr uint64_t kFixDense = 64;

// The warp copies src[lo, hi) to dst[lo, hi), kFixUnr keys per lane in flight.
template <typename K>
__device__ __forceinline__ void warp_copy_keys(K *__restrict__ dst, const K *__restrict__ src, uint32_t lo,
                                               uint32_t hi) {
    const uint32_t lane = threadIdx.x & 31;
    for (uint32_t q = lo; q < hi; q += 32 * kFixUnr) {
        K v[kFixUnr];
#pragma unroll
        for (int r = 0; r < kFixUnr; ++r) {
            const uint32_t x = q + r * 32 + lane;
            if (x < hi) v[r] = __ldcs(src + x);
        }
#pragma unroll
        for (int r = 0; r < kFixUnr; ++r) {
            const uint32_t x = q + r * 32 + lane;
            if (x < hi) dst[x] = v[r];
        }
    }
}

template <class Visit>
__host__ void btree_fix_tile_host(const BtreeStream &S, uint64_t u, Visit &&visit) {
    const uint64_t P0 = u << S.tile_shift, P1 = P0 + S.tile_keys < S.g.n ? P0 + S.tile_keys : S.g.n;
    const uint32_t ru = btree_o_rank(S, u);
    for (uint64_t a = P0; a < P1;) {
        uint32_t lv;
        uint64_t e;
        btree_fix_piece(S, a, P1, lv, e);
        const uint64_t z0 = btree_src_rank_at(S, lv, a) >> S.tile_shift;
        const uint64_t z1 = btree_src_rank_at(S, lv, e - 1) >> S.tile_shift;
        if (z1 - z0 < kFixDense) {
            for (uint64_t z = z0; z <= z1; ++z) {
                if (z == u || btree_o_rank(S, z) > ru) continue;
                uint64_t pa, pe;
                btree_fix_run(S, lv, a, e, z0, z1, z, pa, pe);
                if (pe > pa && !visit(pa, pe - pa)) return;
            }
        } else {
            uint64_t run0 = 0, len = 0;
            for (uint64_t x = a; x < e; ++x) {
                const uint64_t z = btree_src_rank_at(S, lv, x) >> S.tile_shift;
                if (z != u && btree_o_rank(S, z) < ru) {
                    if (!len) run0 = x;
                    ++len;
                } else if (len) {
                    if (!visit(run0, len)) return;
                    len = 0;
                }
            }
            if (len && !visit(run0, len)) return;
        }
        a = e;
    }
}

// Second pass: the scratch ranges still to copy into place.  Range j < h: the
// positions of level j not stored directly (plan R: [max(bnd, start), end);
// plan L: [start, min(bnd, end))); range h (plan L): the last level, from
// scratch[seg1, seg1 + nl) to A[ni, n).  False for an empty range.
struct CopyRange {
    uint64_t dst, src, len;
};

TL_HD int btree_copy_range_count(const BtreeStream &S) { return S.plan == PLAN_O ? 0 : (int)S.g.h + 1; }

TL_HD bool btree_copy_range(const BtreeStream &S, int j, CopyRange &r) {
    const BtreeGeom &g = S.g;
    if (j == (int)g.h) {
        r = CopyRange{g.ni, S.seg1, S.plan == PLAN_L ? g.nl : 0};
        return r.len != 0;
    }
    const uint64_t ls = btree_level_start(g, (uint32_t)j), le = btree_level_end(g, (uint32_t)j), bk = S.bnd[j];
    const uint64_t a = S.plan == PLAN_R ? (bk > ls ? bk : ls) : ls;
    const uint64_t e = S.plan == PLAN_R ? le : (bk < le ? bk : le);
    r = CopyRange{a, a, a < e ? e - a : 0};
    return r.len != 0;
}

// Copy `len` keys src -> dst by the blocks [blk, blk + nblk) of a grid (or one
// block: blk = 0, nblk = 1): 16-byte vectors where src and dst share their
// 16-byte alignment, single keys otherwise and at the ragged ends.  The vectors
// go in block-contiguous chunks of kUnr * blockDim: a block keeps kUnr vectors
// per thread in flight, all from one contiguous stretch, so the DRAM rows it
// touches stay few.  The scratch is read once, so its loads are streaming.
template <typename K, int kUnr = 4>
__device__ __forceinline__ void copy_keys(K *__restrict__ dst, const K *__restrict__ src, uint64_t len,
                                          uint64_t blk, uint64_t nblk) {
    constexpr uint32_t V = 16 / sizeof(K);
    const uint64_t tid = blk * blockDim.x + threadIdx.x;
    const uintptr_t da = reinterpret_cast<uintptr_t>(dst), sa = reinterpret_cast<uintptr_t>(src);
    if (((da ^ sa) & 15) != 0) {
        for (uint64_t x = tid; x < len; x += nblk * blockDim.x) dst[x] = __ldcs(src + x);
        return;
    }
    uint64_t head = ((16 - (da & 15)) & 15) / sizeof(K);
    if (head > len) head = len;
    const uint64_t nvec = (len - head) / V;
    const uint64_t tail0 = head + nvec * V;
    if (tid < head) dst[tid] = __ldcs(src + tid);
    if (tid < len - tail0) dst[tail0 + tid] = __ldcs(src + tail0 + tid);
    uint4 *dv = reinterpret_cast<uint4 *>(dst + head);
    const uint4 *sv = reinterpret_cast<const uint4 *>(src + head);
    const uint64_t chunk = (uint64_t)kUnr * blockDim.x;
    for (uint64_t c0 = blk * chunk; c0 < nvec; c0 += nblk * chunk) {
        uint4 a[kUnr];
#pragma unroll
        for (int u = 0; u < kUnr; ++u) {
            const uint64_t v = c0 + u * blockDim.x + threadIdx.x;
            if (v < nvec) a[u] = __ldcs(sv + v);
        }
#pragma unroll
        for (int u = 0; u < kUnr; ++u) {
            const uint64_t v = c0 + u * blockDim.x + threadIdx.x;
            if (v < nvec) dv[v] = a[u];
        }
    }
}

}  // namespace tl
