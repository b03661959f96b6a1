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
enum BtreePlan { PLAN_R = 0, PLAN_L = 1 };

struct BtreeStream {
    BtreeGeom g;
    FastDiv64 fd;         // b + 1
    FastDiv32 fd32;       // b + 1, for tile-local offsets
    FastDiv32 fd32b;      // b (unused when b = 1)
    uint64_t tile_keys, ntiles;
    uint32_t tile_shift;  // log2(tile_keys)
    int plan;
    uint64_t i2;          // first position of the top tree's last level, (b+1)^(h-1) - 1
    uint64_t E;           // top-tree scratch slots: [0, E)
    uint64_t seg1;        // plan L: scratch slot of final position ni
    uint64_t nscratch;    // scratch slots
    uint64_t bnd[kMaxTopLevels];  // direct-store boundary position of level k
    FastDiv64 pdiv[kMaxTopLevels + 1];  // division by (b+1)^k, k >= 1 (host-built)
};

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
    return S.plan == PLAN_R ? S.ntiles - 1 - t : t;
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
// always tiles with earlier tickets.  False if there are none.
TL_HD bool btree_tile_wait(const BtreeStream &S, uint64_t p0, uint64_t p1, uint64_t &k_lo, uint64_t &k_hi) {
    const BtreeGeom &g = S.g;
    if (S.plan == PLAN_R) {
        if (p0 >= g.lir) return false;
        uint64_t d0 = btree_leaf_dest_bound(S, p0);
        uint64_t d1 = btree_leaf_dest_bound(S, (p1 < g.lir ? p1 : g.lir) - 1) + 1;
        if (d1 > g.n) d1 = g.n;  // a trailing separator bounds past the last leaf key
        uint64_t lo = d0 > p1 ? d0 : p1;
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
    return p < S.g.ni ? p : p - S.g.ni + S.seg1;
}

// Where sorted rank x goes in the stream pass: true -> A[idx] (final position),
// false -> scratch[idx].
TL_HD bool btree_place(const BtreeStream &S, uint64_t x, uint64_t &idx) {
    const uint64_t p = btree_pos(S.g, S.fd, x);
    const bool direct = p >= S.g.ni ? S.plan == PLAN_R : btree_top_direct(S, p);
    idx = direct ? p : btree_scratch_slot(S, p);
    return direct;
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

struct Regime {
    int kind;
    bool to_A;
    uint32_t r0, skip;
    uint64_t dbase;
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
        R.to_A = S.plan == PLAN_R;
        R.dbase = R.to_A ? g.ni + q0 * g.b : S.seg1 + q0 * g.b;
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
        }
    }
    return R;
}

// The tile's groups of top keys (levels kmin.. of each); returns their number.
// Under plan L a tail tile's keys of the top tree's last level are bulk keys.
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

// One level's run of top keys inside a tile.  Level k holds the top ranks with
// c + 1 = x (b+1)^k, x not a multiple of b+1; the t-th such x (t counted from 0
// over the whole level) is x = t + 1 + floor(t / b) and lands at
// btree_level_start(k) + t.  Element e of a run (t = t0 + e) has
// x = xb + e + floor((rb + e) / b), xb the run's first x and rb + 1 its
// remainder mod b+1, and sits at tile offset x * mult - gneg (mult = (b+1)^k f),
// i.e. off0 + (e + floor((rb + e) / b)) * mult with off0 = xb * mult - gneg.
// Offsets are below the tile size, so they are computed modulo 2^32.  Elements
// [0, nlo) of the run (positions below bnd[k]) go to A under plan R and to
// scratch under plan L, the rest the other way round.
struct TopRun {
    uint64_t dest0;
    uint32_t off0, mult, rb, cnt, nlo, pad;
};

// The run of level k of a group of top keys (cnt = 0 when empty).  With hi_k =
// floor(y_hi / (b+1)^k) and lo_k = floor((y_lo - 1) / (b+1)^k), level k holds
// the non-multiples of b+1 in (lo_k, hi_k]: t0 = lo_k - lo_{k+1} of them lie at
// or below lo_k, and (hi_k - hi_{k+1}) - t0 in the range (hi_{k+1} =
// floor(hi_k / (b+1))).  A tile's runs occupy slots s = group * kMaxTopLevels +
// level; slots of levels below kmin or above the tree are empty.
TL_HD TopRun btree_group_run(const BtreeStream &S, const TopGroup &G, uint32_t k) {
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
    const uint64_t bk = S.bnd[k];
    run.nlo = bk <= run.dest0 ? 0 : (bk - run.dest0 < run.cnt ? (uint32_t)(bk - run.dest0) : run.cnt);
    return run;
}

// Tile offset of element e of a run.
TL_HD uint32_t btree_top_item_off(const BtreeStream &S, const TopRun &run, uint32_t e) {
    const uint32_t qe = S.g.b == 1 ? e : S.fd32b.div(run.rb + e);  // b = 1: rb = 0
    return run.off0 + (e + qe) * run.mult;
}

// Does element e of a run go straight to A?
TL_HD bool btree_run_direct(const BtreeStream &S, const TopRun &run, uint32_t e) {
    return (e < run.nlo) == (S.plan == PLAN_R);
}

// Tiles under the direct part of a run (all with earlier tickets, or the tile
// itself); false when the run has no direct part.
TL_HD bool btree_run_wait(const BtreeStream &S, const TopRun &run, uint64_t &k_lo, uint64_t &k_hi) {
    const bool lo_direct = S.plan == PLAN_R;
    const uint32_t e0 = lo_direct ? 0 : run.nlo, e1 = lo_direct ? run.nlo : run.cnt;
    if (e0 >= e1) return false;
    k_lo = (run.dest0 + e0) >> S.tile_shift;
    k_hi = (run.dest0 + e1 - 1) >> S.tile_shift;
    return true;
}

// Shared-memory workspace of btree_stream_tile.
struct TileShared {
    TopRun runs[kMaxTopRuns];
    uint32_t cum[kMaxTopRuns + 1];
    uint32_t nslots;
    int ok;
};

// Warp 0's part of btree_stream_tile: the tile's runs (one lane per slot), their
// prefix sums, and the waits for the tiles under their direct parts.  Kept out
// of line so that its 64-bit state does not crowd the registers of the tile loops.
static __device__ __noinline__ void btree_tile_runs_warp(const BtreeStream &S, uint64_t p0, uint64_t p1,
                                                  unsigned int *flags, Ctrl *ctrl, const WaitCfg &wc,
                                                  TileShared &ts) {
    const uint32_t lane = threadIdx.x;
    TopGroup G0{}, G1{};
    const int ng = btree_stream_groups(S, p0, p1, G0, G1);
    const uint32_t nslots = (uint32_t)ng * kMaxTopLevels;
    uint32_t carry = 0;
    for (uint32_t s0 = 0; s0 < nslots; s0 += 32) {
        const uint32_t sl = s0 + lane;
        TopRun run{};
        if (sl < nslots) run = btree_group_run(S, sl < kMaxTopLevels ? G0 : G1, sl % kMaxTopLevels);
        uint32_t incl = run.cnt;
#pragma unroll
        for (int dd = 1; dd < 32; dd <<= 1) {
            const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, dd);
            if (lane >= (uint32_t)dd) incl += y;
        }
        if (sl < nslots) {
            ts.runs[sl] = run;
            ts.cum[sl] = carry + incl - run.cnt;
        }
        carry += __shfl_sync(0xFFFFFFFFu, incl, 31);
        uint64_t r_lo, r_hi;
        if (run.cnt && btree_run_wait(S, run, r_lo, r_hi))
            for (uint64_t f = r_lo; f <= r_hi; ++f)
                if (!wait_flag(&flags[f], wc.wait_value, ctrl, wc)) ts.ok = 0;
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
// expired (the tile's stores were skipped and the error is recorded).  Warp 0
// computes the tile's runs of top keys (one lane per level) and waits for the
// tiles under their direct parts, while warps 1.. wait for the tiles under the
// bulk keys and store those; then the whole block stores the top keys.
template <typename K>
__device__ __forceinline__ bool btree_stream_tile(const BtreeStream &S, K *__restrict__ A, K *__restrict__ scr,
                                                  unsigned int *flags, Ctrl *ctrl, const WaitCfg &wc, uint64_t k,
                                                  K *sm, TileShared &ts) {
    uint64_t p0, p1;
    btree_tile(S, k, p0, p1);
    if (threadIdx.x == 0) ts.ok = 1;  // the previous tile's readers are past the ticket barrier
    const uint64_t base = load_tile(A, p0, p1, sm);
    publish_read(&flags[k], wc);
    const uint32_t cnt = (uint32_t)(p1 - p0);
    const K *tile = sm + (p0 - base);
    if (threadIdx.x < 32) {
        btree_tile_runs_warp(S, p0, p1, flags, ctrl, wc, ts);
    } else {
        const uint32_t tb = threadIdx.x - 32, nb = blockDim.x - 32;
        uint64_t w_lo, w_hi;
        if (btree_tile_wait(S, p0, p1, w_lo, w_hi))
            for (uint64_t f = w_lo + tb; f <= w_hi; f += nb)
                if (!wait_flag(&flags[f], wc.wait_value, ctrl, wc)) ts.ok = 0;
        bar_sync_tail();
        if (ts.ok) {
            const Regime R = btree_stream_regime(S, p0, p1);
            if (R.kind == 0) {
                for (uint64_t x = p0 + tb; x < p1; x += nb) {
                    if (btree_is_top(S, x)) continue;
                    uint64_t idx;
                    const K key = sm[x - base];
                    if (btree_place(S, x, idx))
                        A[idx] = key;
                    else
                        scr[idx] = key;
                }
            } else if (R.kind == 1) {
                K *tgt = R.to_A ? A : scr;
                const uint32_t d = S.fd32.d;
#pragma unroll 4
                for (uint32_t o = tb; o < cnt; o += nb) {
                    const uint32_t v = R.r0 + o;
                    const uint32_t ql = S.fd32.div(v);
                    if (v - ql * d != R.skip) tgt[R.dbase + (v - ql)] = tile[o];
                }
            }
        }
    }
    __syncthreads();
    if (!ts.ok) return false;
    // top keys, level by level: consecutive threads store consecutive positions
    const uint32_t total = ts.cum[ts.nslots];
    uint32_t r = 0;  // the run of gi only moves forward as gi grows
    for (uint32_t gi = threadIdx.x; gi < total; gi += blockDim.x) {
        while (gi >= ts.cum[r + 1]) ++r;
        const TopRun run = ts.runs[r];
        const uint32_t e = gi - ts.cum[r];
        K *dst = btree_run_direct(S, run, e) ? A : scr;
        dst[run.dest0 + e] = tile[btree_top_item_off(S, run, e)];
    }
    return true;
}

// Second pass: the scratch ranges still to copy into place.  Range j < h: the
// positions of level j not stored directly (plan R: [max(bnd, start), end);
// plan L: [start, min(bnd, end))); range h (plan L): the last level, from
// scratch[seg1, seg1 + nl) to A[ni, n).  False for an empty range.
struct CopyRange {
    uint64_t dst, src, len;
};

TL_HD int btree_copy_range_count(const BtreeStream &S) { return (int)S.g.h + 1; }

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
