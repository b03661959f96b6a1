// B-tree (and BST, b = 1) streaming permutation: schedules, per-tile index
// helpers (shared by the host replay), and the device bodies of the stream and
// scatter passes used by the single-array and the batched kernels.
#pragma once

#include "geometry.cuh"
#include "stream.cuh"

namespace tl {

// Scatter pass: chunks of kScatterChunk scratch slots per CTA work item, taken
// by the block's threads in sub-batches of kScatterUnroll keys per thread.
constexpr int kScatterThreads = 256;
constexpr int kScatterUnroll = 8;
constexpr uint64_t kScatterChunk = 16384;
constexpr int kDeferCap = 32 * kScatterUnroll;  // per-warp queue: one sub-batch never overflows it
static_assert(kScatterChunk <= 65536, "queued chunk offsets are 16-bit");

// ---------------------------------------------------------------- B-tree stream
// Two schedules.  Plan R (right to left): the last level's keys go straight to
// their final positions (they move right), the whole top tree goes through
// scratch.  Plan L (left to right), for trees whose top tree holds most keys:
// the top tree's own last level goes straight to its final positions (those
// keys move left), the last level and the upper top levels go through scratch.
// The host picks the plan with the smaller scratch (the second pass's traffic).
enum BtreePlan { PLAN_R = 0, PLAN_L = 1 };

struct BtreeStream {
    BtreeGeom g;
    FastDiv64 fd;
    FastDiv32 fd32;       // the same divisor b+1, for tile-local offsets
    uint64_t tile_keys, ntiles;
    int plan;
    uint64_t i2;          // plan L: first position of the top tree's last level, (b+1)^(h-1) - 1
    uint64_t ibase;       // plan L: floor(i / (b+1))
    uint64_t nscratch;    // scratch slots
};

TL_HD uint64_t btree_tile_of_ticket(const BtreeStream &S, uint64_t t) {
    return S.plan == PLAN_R ? S.ntiles - 1 - t : t;
}

// Source range of tile k (tiles ascend with position).
TL_HD void btree_tile(const BtreeStream &S, uint64_t k, uint64_t &p0, uint64_t &p1) {
    p0 = k * S.tile_keys;
    p1 = p0 + S.tile_keys < S.g.n ? p0 + S.tile_keys : S.g.n;
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

// Tiles (other than k) whose source lies under the direct destinations of tile
// [p0, p1): right of the tile for plan R, left of it for plan L, i.e. always
// tiles with earlier tickets.  False if there are none.
TL_HD bool btree_tile_wait(const BtreeStream &S, uint64_t p0, uint64_t p1, uint64_t &k_lo, uint64_t &k_hi) {
    const BtreeGeom &g = S.g;
    if (S.plan == PLAN_R) {
        if (p0 >= g.lir) return false;
        uint64_t d0 = btree_leaf_dest_bound(S, p0);
        uint64_t d1 = btree_leaf_dest_bound(S, (p1 < g.lir ? p1 : g.lir) - 1) + 1;
        if (d1 > g.n) d1 = g.n;  // a trailing separator bounds past the last leaf key
        uint64_t lo = d0 > p1 ? d0 : p1;
        if (lo >= d1) return false;
        k_lo = lo / S.tile_keys;
        k_hi = (d1 - 1) / S.tile_keys;
        return true;
    }
    if (p1 <= g.lir) return false;
    uint64_t d0 = btree_top_last_dest_bound(S, p0 > g.lir ? p0 : g.lir);
    uint64_t d1 = btree_top_last_dest_bound(S, p1 - 1) + 1;
    uint64_t hi = d1 < p0 ? d1 : p0;
    if (d0 >= hi) return false;
    k_lo = d0 / S.tile_keys;
    k_hi = (hi - 1) / S.tile_keys;
    return true;
}

// Where sorted rank x goes in the stream pass: true -> A[idx] (final position),
// false -> scratch[idx].
TL_HD bool btree_place(const BtreeStream &S, uint64_t x, uint64_t &idx) {
    const BtreeGeom &g = S.g;
    if (S.plan == PLAN_L) {
        if (x < g.lir) {
            idx = x;
            return false;
        }
        const uint64_t c = x - g.l - g.r;
        uint64_t q, rem;
        S.fd.divmod(c + 1, q, rem);
        if (rem != 0) {
            idx = S.i2 + c - q;
            return true;
        }
        idx = g.lir + q - 1 - S.ibase;
        return false;
    }
    if (x < g.l + g.i) {
        uint64_t j, t;
        S.fd.divmod(x, j, t);
        if (t < g.b) {
            idx = g.ni + j * g.b + t;
            return true;
        }
        idx = j;
        return false;
    }
    if (x < g.lir) {
        idx = g.ni + x - g.i;
        return true;
    }
    idx = x - g.l - g.r;
    return false;
}

// Tile-local form of btree_place: the one 64-bit division by b+1 per tile is done
// at the tile's first divided rank x0; each key then divides a small 32-bit
// offset.  Same result as btree_place for every x >= p0 of the tile.
struct TileDiv {
    uint64_t x0, q0;  // first rank that needs the division, and its quotient
    uint32_t r0;      // and its remainder
};

TL_HD TileDiv btree_tile_div(const BtreeStream &S, uint64_t p0) {
    TileDiv td;
    uint64_t v;
    if (S.plan == PLAN_L) {
        td.x0 = p0 > S.g.lir ? p0 : S.g.lir;
        v = td.x0 - S.g.l - S.g.r + 1;  // c + 1
    } else {
        td.x0 = p0;
        v = p0;
    }
    uint64_t r;
    S.fd.divmod(v, td.q0, r);
    td.r0 = (uint32_t)r;
    return td;
}

TL_HD bool btree_place_tile(const BtreeStream &S, const TileDiv &td, uint64_t x, uint64_t &idx) {
    const BtreeGeom &g = S.g;
    if (S.plan == PLAN_L) {
        if (x < g.lir) {
            idx = x;
            return false;
        }
        const uint32_t v = td.r0 + (uint32_t)(x - td.x0);
        const uint32_t ql = S.fd32.div(v);
        const uint32_t rem = v - ql * (uint32_t)S.fd32.d;
        const uint64_t q = td.q0 + ql;
        if (rem != 0) {
            idx = S.i2 + (x - g.l - g.r) - q;
            return true;
        }
        idx = g.lir + q - 1 - S.ibase;
        return false;
    }
    if (x < g.l + g.i) {
        const uint32_t v = td.r0 + (uint32_t)(x - td.x0);
        const uint32_t ql = S.fd32.div(v);
        const uint32_t t = v - ql * (uint32_t)S.fd32.d;
        const uint64_t j = td.q0 + ql;
        if (t < g.b) {
            idx = g.ni + j * g.b + t;
            return true;
        }
        idx = j;
        return false;
    }
    if (x < g.lir) {
        idx = g.ni + x - g.i;
        return true;
    }
    idx = x - g.l - g.r;
    return false;
}

// Per-tile fast paths.  Inside most tiles every key follows one rule: with
// v = r0 + o (o = x - p0, r0 a remainder fixed per tile) and ql = v / (b+1),
// rem = v - ql (b+1), the key goes to A[dbase + v - ql] unless rem == skip, in
// which case it goes to scratch[sbase + ql] (kind 1); or every key goes to
// scratch[sbase + o] (kind 2).  kind 0: the tile straddles a boundary, use the
// generic per-key form.  Derivations: plan R last level, idx = ni + j b + t with
// j = q0 + ql, t = rem, so dbase = ni + q0 b; plan L top-last level, idx =
// i2 + c - q with c + 1 = v + q0 (b+1) - r0 ..., so dbase = i2 + c0 - q0 - r0.
struct Regime {
    uint64_t dbase, sbase;
    uint32_t r0, skip;
    int kind;
    // scatter only: second-level fast path for the keys with rem == skip (one
    // level up): their index m = q0 + ql + madd, written m = Q1 (b+1) + R1 +
    // ql, lands at d2base + m - m / (b+1) when m % (b+1) != 0.
    uint64_t Q1, d2base;
    uint32_t R1;
    int two;
};

TL_HD Regime btree_stream_regime(const BtreeStream &S, uint64_t p0, uint64_t p1) {
    const BtreeGeom &g = S.g;
    Regime R{0, 0, 0, 0, 0, 0, 0, 0, 0};
    uint64_t q0, r0;
    if (S.plan == PLAN_L) {
        if (p0 >= g.lir) {
            const uint64_t c0 = p0 - g.l - g.r;
            S.fd.divmod(c0 + 1, q0, r0);
            R.kind = 1;
            R.r0 = (uint32_t)r0;
            R.skip = 0;
            R.dbase = S.i2 + c0 - q0 - r0;
            R.sbase = g.lir + q0 - 1 - S.ibase;
        } else if (p1 <= g.lir) {
            R.kind = 2;
            R.sbase = p0;
        }
    } else {
        if (p1 <= g.l + g.i) {
            S.fd.divmod(p0, q0, r0);
            R.kind = 1;
            R.r0 = (uint32_t)r0;
            R.skip = (uint32_t)g.b;
            R.dbase = g.ni + q0 * g.b;
            R.sbase = q0;
        } else if (p0 >= g.lir) {
            R.kind = 2;
            R.sbase = p0 - g.l - g.r;
        }
    }
    return R;
}

// Regime form of btree_place for offset o of a kind-1 or kind-2 tile.
TL_HD bool btree_regime_place(const BtreeStream &S, const Regime &R, uint32_t o, uint64_t &idx) {
    if (R.kind == 2) {
        idx = R.sbase + o;
        return false;
    }
    const uint32_t v = R.r0 + o;
    const uint32_t ql = S.fd32.div(v);
    const uint32_t rem = v - ql * S.fd32.d;
    if (rem != R.skip) {
        idx = R.dbase + (v - ql);
        return true;
    }
    idx = R.sbase + ql;
    return false;
}

// Scatter-chunk fast path: slots of the chunk whose destination follows
// dest = dbase + v - ql (v = r0 + o) unless rem == skip (those take the
// generic btree_slot_dest).  kind 0: generic for the whole chunk.
TL_HD Regime btree_scatter_regime(const BtreeStream &S, uint64_t c0, uint64_t c1) {
    const BtreeGeom &g = S.g;
    Regime R{0, 0, 0, 0, 0, 0, 0, 0, 0};
    uint64_t q0, r0, Q1, R1;
    // The keys with rem == skip sit one level up.  With m their index within
    // the runs of that level (1-based, m = q0 + ql + madd), the ones with
    // m % (b+1) != 0 sit at level L2 of the top tree at pw[L2] - 1 + (m - m/(b+1))
    // - 1 + ... : d2base + m - floor(m/(b+1)).
    auto second = [&](uint64_t mfirst, uint32_t level_from_root) {
        if (level_from_root >= 48) return;
        S.fd.divmod(mfirst, Q1, R1);
        R.Q1 = Q1;
        R.R1 = (uint32_t)R1;
        R.d2base = g.pw[level_from_root] - 2;
        R.two = 1;
    };
    if (S.plan == PLAN_R) {
        if (g.h >= 1) {
            S.fd.divmod(c0 + 1, q0, r0);
            R.kind = 1;
            R.r0 = (uint32_t)r0;
            R.skip = 0;
            R.dbase = g.pw[g.h - 1] - 2 + q0 * g.b;
            // rem == 0: c + 1 = M (b+1), M = q0 + ql; level h-2 when M % (b+1) != 0
            if (g.h >= 2) second(q0, g.h - 2);
        }
    } else if (c1 <= g.l + g.i) {
        S.fd.divmod(c0, q0, r0);
        R.kind = 1;
        R.r0 = (uint32_t)r0;
        R.skip = (uint32_t)g.b;
        R.dbase = g.ni + q0 * g.b;
        // separator of leaf j = q0 + ql: top rank j, c + 1 = j + 1; level h-1
        // (the top tree's last level) when (j+1) % (b+1) != 0
        if (g.h >= 1) second(q0 + 1, g.h - 1);
    } else if (c0 >= g.lir && g.h >= 2) {
        S.fd.divmod(c0 - g.lir + S.ibase + 1, q0, r0);
        R.kind = 1;
        R.r0 = (uint32_t)r0;
        R.skip = 0;
        R.dbase = g.pw[g.h - 2] - 2 + q0 * g.b;
        // mr == 0: M = (mq)(b+1), mq = q0 + ql; level h-3 when mq % (b+1) != 0
        if (g.h >= 3) second(q0, g.h - 3);
    }
    return R;
}

// Final position of the key held by scratch slot `slot`.
TL_HD uint64_t btree_slot_dest(const BtreeStream &S, uint64_t slot) {
    const BtreeGeom &g = S.g;
    if (S.plan == PLAN_R) return btree_perfect_pos(g, S.fd, slot, g.h);
    uint64_t s;
    if (slot < g.lir) {
        s = slot;
    } else {
        const uint64_t M = slot - g.lir + S.ibase + 1;
        s = M * (g.b + 1) - 1 + g.l + g.r;
    }
    return btree_pos(g, S.fd, s);
}

// Destination of scratch slot c0 + o under a kind-1 scatter regime (the
// generic btree_slot_dest only for keys two or more levels above the fast one).
TL_HD uint64_t btree_regime_slot_dest(const BtreeStream &S, const Regime &R, uint64_t c0, uint32_t o) {
    const uint32_t d = S.fd32.d;
    const uint32_t vv = R.r0 + o;
    const uint32_t ql = S.fd32.div(vv);
    if (vv - ql * d != R.skip) return R.dbase + (vv - ql);
    if (R.two) {
        const uint32_t w = R.R1 + ql;
        const uint32_t q2 = S.fd32.div(w);
        const uint32_t r2 = w - q2 * d;
        if (r2 != 0) {
            // m = Q1 (b+1) + w = (Q1 + q2)(b+1) + r2: pos = pw[L] - 1 + (Q1+q2) b + r2 - 1
            return R.d2base + (R.Q1 + q2) * S.g.b + r2;
        }
    }
    return btree_slot_dest(S, c0 + o);
}


// Tile-local form of btree_slot_dest for the slots of a chunk starting at c0:
// the division of the chunk's first slot is done once, each slot then divides a
// small offset, and only keys two or more levels above the direct level take
// the generic path.  Same result as btree_slot_dest for every slot >= c0.
struct ScatterDiv {
    uint64_t c0, q0, ubase, uq0;
    uint32_t r0, ur0;
};

TL_HD ScatterDiv btree_scatter_div(const BtreeStream &S, uint64_t c0) {
    ScatterDiv sd;
    uint64_t r;
    sd.c0 = c0;
    if (S.plan == PLAN_R) {
        S.fd.divmod(c0 + 1, sd.q0, r);
        sd.r0 = (uint32_t)r;
        sd.ubase = sd.uq0 = 0;
        sd.ur0 = 0;
        return sd;
    }
    S.fd.divmod(c0, sd.q0, r);
    sd.r0 = (uint32_t)r;
    sd.ubase = c0 > S.g.lir ? c0 : S.g.lir;
    S.fd.divmod(sd.ubase - S.g.lir + S.ibase + 1, sd.uq0, r);
    sd.ur0 = (uint32_t)r;
    return sd;
}

TL_HD uint64_t btree_slot_dest_tile(const BtreeStream &S, const ScatterDiv &sd, uint64_t slot) {
    const BtreeGeom &g = S.g;
    const uint32_t d = S.fd32.d;
    if (S.plan == PLAN_R) {  // slot = top rank c; c + 1 = q (b+1) + rem
        const uint32_t v = sd.r0 + (uint32_t)(slot - sd.c0);
        const uint32_t ql = S.fd32.div(v), rem = v - ql * d;
        if (rem != 0) return g.pw[g.h - 1] - 1 + (sd.q0 + ql) * g.b + rem - 1;
        return btree_perfect_pos(g, S.fd, slot, g.h);
    }
    if (slot < g.lir) {  // sorted rank s = slot: last level, or a separator
        if (slot >= g.l + g.i) return g.ni + slot - g.i;
        const uint32_t v = sd.r0 + (uint32_t)(slot - sd.c0);
        const uint32_t ql = S.fd32.div(v), t = v - ql * d;
        const uint64_t j = sd.q0 + ql;
        if (t < g.b) return g.ni + j * g.b + t;
        return btree_perfect_pos(g, S.fd, j, g.h);
    }
    // upper top keys: c + 1 = M (b+1), M = slot - lir + ibase + 1 = Mq (b+1) + Mr
    const uint32_t v = sd.ur0 + (uint32_t)(slot - sd.ubase);
    const uint32_t ql = S.fd32.div(v), mr = v - ql * d;
    const uint64_t mq = sd.uq0 + ql;
    if (mr != 0) return g.pw[g.h - 2] - 1 + mq * g.b + mr - 1;
    return btree_perfect_pos(g, S.fd, (mq * d) * d - 1, g.h);
}

TL_HD void btree_choose_plan(BtreeStream &S) {
    const BtreeGeom &g = S.g;
    S.plan = PLAN_R;
    S.nscratch = g.ni;
    if (g.h < 1) return;
    const uint64_t i2 = g.pw[g.h - 1] - 1;
    const uint64_t ibase = g.i / (g.b + 1);
    // Plan L needs every direct key to move left: i2 <= l + r + floor((c+1)/(b+1))
    // at the smallest trailing top rank c = i.
    if (g.lir >= g.n) return;
    if (i2 > g.l + g.r + (g.i + 1) / (g.b + 1)) return;
    const uint64_t upper = g.ni / (g.b + 1) - ibase;
    const uint64_t nscr = g.lir + upper;
    if (nscr < g.ni) {
        S.plan = PLAN_L;
        S.i2 = i2;
        S.ibase = ibase;
        S.nscratch = nscr;
    }
}

// Stream pass for tile k of one array (block-wide).  False if a bounded wait
// expired (the tile's stores were skipped and the error is recorded).
template <typename K>
__device__ __forceinline__ bool btree_stream_tile(const BtreeStream &S, K *__restrict__ A, K *__restrict__ scr,
                                                  unsigned int *flags, Ctrl *ctrl, const WaitCfg &wc, uint64_t k,
                                                  K *sm, int *s_ok) {
    uint64_t p0, p1;
    btree_tile(S, k, p0, p1);
    const uint64_t base = load_tile(A, p0, p1, sm);
    publish_read(&flags[k], wc);
    uint64_t k_lo, k_hi;
    if (btree_tile_wait(S, p0, p1, k_lo, k_hi) &&
        !wait_tiles(flags, (long long)k_lo, (long long)k_hi, ctrl, wc, s_ok))
        return false;
    const Regime R = btree_stream_regime(S, p0, p1);
    const uint32_t cnt = (uint32_t)(p1 - p0);
    const K *tile = sm + (p0 - base);
    if (R.kind == 1) {
        const uint32_t d = S.fd32.d;
#pragma unroll 4
        for (uint32_t o = threadIdx.x; o < cnt; o += blockDim.x) {
            const K key = tile[o];
            const uint32_t v = R.r0 + o;
            const uint32_t ql = S.fd32.div(v);
            if (v - ql * d != R.skip)
                A[R.dbase + (v - ql)] = key;
            else
                scr[R.sbase + ql] = key;
        }
    } else if (R.kind == 2) {
        K *dst = scr + R.sbase;
#pragma unroll 4
        for (uint32_t o = threadIdx.x; o < cnt; o += blockDim.x) dst[o] = tile[o];
    } else {
        const TileDiv td = btree_tile_div(S, p0);
        for (uint64_t x = p0 + threadIdx.x; x < p1; x += blockDim.x) {
            uint64_t idx;
            const K key = sm[x - base];
            if (btree_place_tile(S, td, x, idx))
                A[idx] = key;
            else
                scr[idx] = key;
        }
    }
    return true;
}

// Scratch -> final positions for the chunk of kScatterChunk slots at c0.
// Every thread first issues kScatterUnroll coalesced loads (scratch is read
// through L2 only), then stores.  Under a kind-1 regime the keys on the fast
// path are stored directly; the others (one level up and above, at most one in
// b+1) are queued per warp in shared memory and placed afterwards by the whole
// warp, so their longer path runs on full warps instead of diverging every
// step.  Binary trees (b = 1) use the branch-free trailing-zeros position.
// `qval`/`qoff` hold kDeferCap (value, chunk offset) entries per warp of the
// block; binary trees never touch them.  kBinaryOnly: the caller guarantees a
// binary tree under plan R, and only the trailing-zeros path is compiled.
template <typename K, bool kBinaryOnly = false>
__device__ __forceinline__ void btree_scatter_chunk(const BtreeStream &S, K *__restrict__ A,
                                                    const K *__restrict__ scr, uint64_t c0, K *qval,
                                                    uint16_t *qoff) {
    const uint64_t c1 = min(S.nscratch, c0 + kScatterChunk);
    const uint32_t cnt = (uint32_t)(c1 - c0);
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    K *wq = qval + warp * kDeferCap;
    uint16_t *wo = qoff + warp * kDeferCap;
    const bool binary = kBinaryOnly || (S.g.b == 1 && S.plan == PLAN_R);
    const Regime R = binary ? Regime{} : btree_scatter_regime(S, c0, c1);
    const ScatterDiv sd = (binary || R.kind == 1) ? ScatterDiv{} : btree_scatter_div(S, c0);
    const uint32_t d = S.fd32.d;
    for (uint32_t sub = 0; sub < cnt; sub += blockDim.x * kScatterUnroll) {
        K v[kScatterUnroll];
#pragma unroll
        for (int u = 0; u < kScatterUnroll; ++u) {
            const uint32_t o = sub + threadIdx.x + u * blockDim.x;
            if (o < cnt) v[u] = __ldcg(scr + c0 + o);
        }
        if (binary) {
#pragma unroll
            for (int u = 0; u < kScatterUnroll; ++u) {
                const uint32_t o = sub + threadIdx.x + u * blockDim.x;
                if (o < cnt) A[btree_perfect_pos(S.g, S.fd, c0 + o, S.g.h)] = v[u];
            }
        } else if (R.kind == 1) {
            uint32_t nq = 0;  // warp-uniform
#pragma unroll
            for (int u = 0; u < kScatterUnroll; ++u) {
                const uint32_t o = sub + threadIdx.x + u * blockDim.x;
                bool defer = false;
                if (o < cnt) {
                    const uint32_t vv = R.r0 + o;
                    const uint32_t ql = S.fd32.div(vv);
                    if (vv - ql * d != R.skip)
                        A[R.dbase + (vv - ql)] = v[u];
                    else
                        defer = true;
                }
                const unsigned m = __ballot_sync(0xFFFFFFFFu, defer);
                if (defer) {
                    const uint32_t at = nq + __popc(m & ((1u << lane) - 1u));
                    wq[at] = v[u];
                    wo[at] = (uint16_t)o;
                }
                nq += __popc(m);
            }
            __syncwarp();
            for (uint32_t e = lane; e < nq; e += 32) A[btree_regime_slot_dest(S, R, c0, wo[e])] = wq[e];
            __syncwarp();
        } else {
#pragma unroll
            for (int u = 0; u < kScatterUnroll; ++u) {
                const uint32_t o = sub + threadIdx.x + u * blockDim.x;
                if (o < cnt) A[btree_slot_dest_tile(S, sd, c0 + o)] = v[u];
            }
        }
    }
}

}  // namespace tl
