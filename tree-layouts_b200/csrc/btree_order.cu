// Plan O's tile order for the B-tree / BST stream pass, and its per-geometry cache.
//
// The stream pass stores a key straight into its final position only when the
// tile under that position was read before the key's own tile; every other key
// takes a second trip through scratch.  With tiles in position order (plans R
// and L) the keys of whole levels go the wrong way: for a BST about 39 % of all
// keys, for a B-tree with b = 16 and n = 2^30 about 38 %.  Here each tile u
// names the tile that feeds it the most keys (pred(u), when that run holds at
// least tile_keys / 8 of them) and gets the depth m(u) = 1 + m(pred(u)) of that
// chain (0 without a pred, kChainCap on a cycle).  Tiles go in decreasing m, so
// the heaviest edge into every tile points forward in the order and the chains
// of leaf edges (and of the top tree's heavy levels) stay consistent; ties go
// right to left or left to right, whichever leaves fewer scratch keys.  For
// 8-byte keys this leaves 6.1 % of the keys of a b = 16 B-tree of 5e8 keys, 6.5 %
// at 2^30 keys, 10 % of a b = 8 tree of 6e7 keys and 20 % of a BST of 2^30 - 1
// keys for the second pass.
//
// The tables depend on (n, b, tile_keys) only.  They are computed once per
// process (O(tiles): a few source runs per tile) and copied once to each device
// that uses them.  A permutation computes them with its two per-tile passes as
// kernels on its own stream (btree_order_prepare; the BST of 2^30 - 1 keys
// took 115 ms with them on 8 host threads); other callers, and a permutation
// whose kernels cannot run, compute them on the host's threads.  Host and
// device copies live until the process exits.  A geometry seen for the first
// time while its stream is being captured gets no device copy (the permutation
// then takes plan R or L).
#include <algorithm>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "btree_order.h"
#include "bulk.cuh"
#include "internal.h"

namespace tl {

constexpr uint32_t kChainCap = 64;
constexpr size_t kMaxOrderEntries = 64;
constexpr int kMaxOrderDevices = 64;

static void order_preds_range(const BtreeStream &S, std::vector<int64_t> &pred, uint64_t u0, uint64_t u1);

// fn(u0, u1) over [0, N) in contiguous slices on the host's threads (one
// slice per 4096 tiles at most, 16 threads at most).
template <typename Fn>
static void parallel_tiles(uint64_t N, Fn fn) {
    const uint64_t hw = std::max(1u, std::thread::hardware_concurrency());
    const uint64_t T = std::max<uint64_t>(1, std::min<uint64_t>({hw, 16, (N + 4095) / 4096}));
    if (T == 1) {
        fn(0, N);
        return;
    }
    std::vector<std::thread> th;
    th.reserve(T);
    for (uint64_t t = 0; t < T; ++t) th.emplace_back(fn, N * t / T, N * (t + 1) / T);
    for (auto &x : th) x.join();
}

// pred(u) for every tile: the source tile with the longest run into u.
static void order_preds(const BtreeStream &S, std::vector<int64_t> &pred) {
    const uint64_t N = S.ntiles;
    pred.assign(N, -1);
    parallel_tiles(N, [&](uint64_t u0, uint64_t u1) { order_preds_range(S, pred, u0, u1); });
}

// pred(u): the source tile with the longest run into tile u, if that run holds
// at least tile_keys / 8 keys, else -1.
TL_HD int64_t order_pred_of(const BtreeStream &S, uint64_t u) {
    const uint64_t T = S.tile_keys, thr = T / 8;
    const uint64_t P0 = u << S.tile_shift, P1 = P0 + T < S.g.n ? P0 + T : S.g.n;
    uint64_t best = 0;
    int64_t bz = -1;
    for (uint64_t a = P0; a < P1;) {
        uint32_t lv;
        uint64_t e;
        btree_fix_piece(S, a, P1, lv, e);
        if (e - a >= thr) {
            const uint64_t z0 = btree_src_rank(S, a) >> S.tile_shift;
            const uint64_t z1 = btree_src_rank(S, e - 1) >> S.tile_shift;
            if (z1 - z0 <= 64)  // more runs than that are all shorter than thr
                for (uint64_t z = z0; z <= z1; ++z) {
                    if (z == u) continue;
                    uint64_t pa, pe;
                    btree_fix_run(S, lv, a, e, z0, z1, z, pa, pe);
                    if (pe - pa > best) {
                        best = pe - pa;
                        bz = (int64_t)z;
                    }
                }
        }
        a = e;
    }
    return best >= thr ? bz : -1;
}

static void order_preds_range(const BtreeStream &S, std::vector<int64_t> &pred, uint64_t u0, uint64_t u1) {
    for (uint64_t u = u0; u < u1; ++u) pred[u] = order_pred_of(S, u);
}

// Scratch keys of tile u under the ticket table tab: the count of the runs
// btree_fix_tile_host visits (same two cases), by the lanes of one warp (each
// takes every 32nd source tile of a piece, or every 32nd position of a dense
// piece); the caller adds the lanes' parts.
__device__ uint32_t order_tile_scratch(const BtreeStream &S, const uint2 *__restrict__ tab, uint64_t u,
                                       uint32_t lane) {
    const uint64_t P0 = u << S.tile_shift, P1 = P0 + S.tile_keys < S.g.n ? P0 + S.tile_keys : S.g.n;
    const uint32_t ru = __ldg(tab + u).x;
    uint32_t c = 0;
    for (uint64_t a = P0; a < P1;) {
        uint32_t lv;
        uint64_t e;
        btree_fix_piece(S, a, P1, lv, e);
        const uint64_t z0 = btree_src_rank_at(S, lv, a) >> S.tile_shift;
        const uint64_t z1 = btree_src_rank_at(S, lv, e - 1) >> S.tile_shift;
        if (z1 - z0 < kFixDense) {
            for (uint64_t z = z0 + lane; z <= z1; z += 32) {
                if (z == u || __ldg(tab + z).x > ru) continue;
                uint64_t pa, pe;
                btree_fix_run(S, lv, a, e, z0, z1, z, pa, pe);
                c += (uint32_t)(pe - pa);
            }
        } else {
            for (uint64_t x = a + lane; x < e; x += 32) {
                const uint64_t z = btree_src_rank_at(S, lv, x) >> S.tile_shift;
                c += z != u && __ldg(tab + z).x < ru;
            }
        }
        a = e;
    }
    return c;
}

__global__ void order_pred_kernel(const BtreeStream S, int32_t *__restrict__ pred) {
    for (uint64_t u = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; u < S.ntiles;
         u += (uint64_t)gridDim.x * blockDim.x)
        pred[u] = (int32_t)order_pred_of(S, u);
}

// Scratch keys per tile under two ticket tables, a warp per tile.
__global__ void order_scratch_kernel(const BtreeStream S, const uint2 *__restrict__ ta, const uint2 *__restrict__ tb,
                                     uint32_t *__restrict__ ca, uint32_t *__restrict__ cb) {
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t warps = (uint64_t)gridDim.x * (blockDim.x >> 5);
    for (uint64_t u = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; u < S.ntiles; u += warps) {
        const uint32_t a = __reduce_add_sync(0xFFFFFFFFu, order_tile_scratch(S, ta, u, lane));
        const uint32_t b = __reduce_add_sync(0xFFFFFFFFu, order_tile_scratch(S, tb, u, lane));
        if (lane == 0) {
            ca[u] = a;
            cb[u] = b;
        }
    }
}

// Tickets by decreasing chain depth m (counting sort), ties in position order
// (asc) or against it.
static void order_tickets(uint64_t N, const std::vector<uint8_t> &m, bool asc, OrderVectors &v) {
    std::vector<uint64_t> start(kChainCap + 1, 0);
    for (uint64_t u = 0; u < N; ++u) ++start[m[u]];
    uint64_t acc = 0;
    for (int mm = (int)kChainCap; mm >= 0; --mm) {
        const uint64_t c = start[mm];
        start[mm] = acc;
        acc += c;
    }
    v.tab.assign(N, make_uint2(0, kNoSlot));
    v.order.assign(N, 0);
    for (uint64_t i = 0; i < N; ++i) {
        const uint64_t u = asc ? i : N - 1 - i;
        const uint64_t t = start[m[u]]++;
        v.order[t] = (uint32_t)u;
        v.tab[u].x = (uint32_t)t;
    }
}

// Given each tile's scratch keys under v's tickets: the tiles that receive
// scratch keys, each given a tile of scratch; the runs of whole scratch tiles
// for the bulk-copy engine; the fix pass's segments for the rest.  Returns the
// number of scratch keys.
static uint64_t order_finish(BtreeStream S, const std::vector<uint32_t> &cnt, OrderVectors &v) {
    const uint64_t N = S.ntiles;
    S.tab = v.tab.data();
    std::vector<uint8_t> full(N, 0);
    uint64_t keys = 0, slots = 0;
    for (uint64_t u = 0; u < N; ++u) {
        const uint64_t c = cnt[u];
        if (!c) continue;
        keys += c;
        v.tab[u].y = (uint32_t)slots++;
        full[u] = c == std::min<uint64_t>(S.tile_keys, S.g.n - (u << S.tile_shift));
    }
    v.scratch_tiles = slots;
    // runs of consecutive full tiles (their slots are consecutive too): the
    // longest go to the bulk-copy engine
    std::vector<uint4> runs;
    for (uint64_t u = 0; u < N;) {
        if (!full[u]) {
            ++u;
            continue;
        }
        uint64_t w = u;
        while (w < N && full[w]) ++w;
        runs.push_back(make_uint4((uint32_t)u, (uint32_t)w, v.tab[u].y, 0));
        u = w;
    }
    std::stable_sort(runs.begin(), runs.end(), [](uint4 a, uint4 b) { return a.y - a.x > b.y - b.x; });
    if (runs.size() > (size_t)kMaxBulkRanges) runs.resize(kMaxBulkRanges);
    std::sort(runs.begin(), runs.end(), [](uint4 a, uint4 b) { return a.x < b.x; });
    v.ranges = runs;
    std::vector<uint8_t> bulk(N, 0);
    for (const uint4 &r : runs)
        for (uint32_t u = r.x; u < r.y; ++u) bulk[u] = 1;
    // the fix pass's copies: the scratch runs of the other tiles, adjacent ones merged
    v.segs.clear();
    for (uint64_t u = 0; u < N; ++u) {
        if (v.tab[u].y == kNoSlot || bulk[u]) continue;
        const int64_t so = btree_o_soff(S, u);
        btree_fix_tile_host(S, u, [&](uint64_t pa, uint64_t len) {
            const uint64_t src = pa + (uint64_t)so;
            if (!v.segs.empty()) {
                FixSeg &l = v.segs.back();
                const uint64_t ld = l.dst_len & kSegDstMask, ll = l.dst_len >> 48;
                if (ld + ll == pa && l.src + ll == src && ll + len <= kFixSegMax) {
                    l.dst_len = ld | ((ll + len) << 48);
                    return true;
                }
            }
            v.segs.push_back(FixSeg{pa | (len << 48), src});
            return true;
        });
    }
    return keys;
}

// Tickets in one tie order, the tiles' scratch counts on the host's threads,
// and the rest of the tables.
static uint64_t order_by_depth(BtreeStream S, const std::vector<uint8_t> &m, bool asc, OrderVectors &v) {
    const uint64_t N = S.ntiles;
    order_tickets(N, m, asc, v);
    S.tab = v.tab.data();
    std::vector<uint32_t> cnt(N, 0);
    parallel_tiles(N, [&](uint64_t u0, uint64_t u1) {
        for (uint64_t u = u0; u < u1; ++u) {
            uint64_t c = 0;
            btree_fix_tile_host(S, u, [&](uint64_t, uint64_t len) {
                c += len;
                return true;
            });
            cnt[u] = (uint32_t)c;
        }
    });
    return order_finish(S, cnt, v);
}

// Chain depths m(u) = 1 + m(pred(u)) (0 without a pred, kChainCap on a
// cycle), each path walked once (state 1: on the current path).
static void order_chains(uint64_t N, const std::vector<int64_t> &pred, std::vector<uint8_t> &m) {
    m.assign(N, 0);
    std::vector<uint8_t> state(N, 0);
    std::vector<uint64_t> path;
    for (uint64_t u = 0; u < N; ++u) {
        if (state[u] == 2) continue;
        path.clear();
        int64_t w = (int64_t)u;
        while (w >= 0 && state[w] == 0) {
            state[w] = 1;
            path.push_back((uint64_t)w);
            w = pred[w];
        }
        uint32_t cur = w < 0 ? 0 : state[w] == 1 ? kChainCap : std::min<uint32_t>(kChainCap, 1u + m[w]);
        for (size_t j = path.size(); j-- > 0;) {
            m[path[j]] = (uint8_t)cur;
            state[path[j]] = 2;
            cur = std::min<uint32_t>(kChainCap, cur + 1);
        }
    }
}

void btree_compute_order(const BtreeStream &S0, OrderVectors &v) {
    BtreeStream S = S0;
    S.plan = PLAN_O;
    const uint64_t N = S.ntiles;
    std::vector<int64_t> pred;
    order_preds(S, pred);
    std::vector<uint8_t> m;
    order_chains(N, pred, m);
    // both tie orders (right to left, left to right), side by side; keep the
    // one with fewer scratch keys (right to left on a tie)
    OrderVectors w0, w1;
    uint64_t c0 = 0, c1 = 0;
    std::thread t1([&] { c1 = order_by_depth(S, m, true, w1); });
    c0 = order_by_depth(S, m, false, w0);
    t1.join();
    std::swap(v, c1 < c0 ? w1 : w0);
}

// The same tables with the two per-tile passes (pred, and the scratch counts
// under both tie orders) run as kernels on st; the chain walk, the tickets
// and the rest stay on the host.  False (nothing cached) on any CUDA failure.
bool btree_compute_order_device(const BtreeStream &S0, cudaStream_t st, OrderVectors &v) {
    BtreeStream S = S0;
    S.plan = PLAN_O;
    const uint64_t N = S.ntiles;
    const size_t b_pred = (N * 4 + 255) / 256 * 256, b_tab = (N * 8 + 255) / 256 * 256, b_cnt = b_pred;
    char *buf = static_cast<char *>(workspace_acquire(b_pred + 2 * b_tab + 2 * b_cnt));
    if (!buf) return false;
    int32_t *d_pred = reinterpret_cast<int32_t *>(buf);
    uint2 *d_ta = reinterpret_cast<uint2 *>(buf + b_pred), *d_tb = reinterpret_cast<uint2 *>(buf + b_pred + b_tab);
    uint32_t *d_ca = reinterpret_cast<uint32_t *>(buf + b_pred + 2 * b_tab);
    uint32_t *d_cb = reinterpret_cast<uint32_t *>(buf + b_pred + 2 * b_tab + b_cnt);
    const unsigned grid = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((N + 127) / 128, 1u << 20));
    bool ok = true;
    std::vector<int32_t> p32(N);
    order_pred_kernel<<<grid, 128, 0, st>>>(S, d_pred);
    ok = cudaMemcpyAsync(p32.data(), d_pred, N * 4, cudaMemcpyDeviceToHost, st) == cudaSuccess &&
         cudaStreamSynchronize(st) == cudaSuccess;
    OrderVectors w0, w1;
    std::vector<uint32_t> n0(N), n1(N);
    if (ok) {
        std::vector<int64_t> pred(p32.begin(), p32.end());
        std::vector<uint8_t> m;
        order_chains(N, pred, m);
        order_tickets(N, m, false, w0);
        order_tickets(N, m, true, w1);
        ok = cudaMemcpyAsync(d_ta, w0.tab.data(), N * 8, cudaMemcpyHostToDevice, st) == cudaSuccess &&
             cudaMemcpyAsync(d_tb, w1.tab.data(), N * 8, cudaMemcpyHostToDevice, st) == cudaSuccess;
        const unsigned wgrid = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((N + 7) / 8, 1u << 20));
        if (ok) order_scratch_kernel<<<wgrid, 256, 0, st>>>(S, d_ta, d_tb, d_ca, d_cb);
        ok = ok && cudaMemcpyAsync(n0.data(), d_ca, N * 4, cudaMemcpyDeviceToHost, st) == cudaSuccess &&
             cudaMemcpyAsync(n1.data(), d_cb, N * 4, cudaMemcpyDeviceToHost, st) == cudaSuccess &&
             cudaStreamSynchronize(st) == cudaSuccess && cudaGetLastError() == cudaSuccess;
    }
    if (!ok) {
        cudaGetLastError();
        cudaStreamSynchronize(st);
        cudaGetLastError();
    }
    workspace_release(buf);
    if (!ok) return false;
    uint64_t c0 = 0, c1 = 0;
    for (uint64_t u = 0; u < N; ++u) {
        c0 += n0[u];
        c1 += n1[u];
    }
    const bool ltr = c1 < c0;  // right to left on a tie
    order_finish(S, ltr ? n1 : n0, ltr ? w1 : w0);
    std::swap(v, ltr ? w1 : w0);
    return true;
}

namespace {
struct OrderEntry {
    uint64_t n, b, tile_keys;
    OrderVectors v;
    void *dev[kMaxOrderDevices] = {};  // segs, then tab and order
};
std::mutex g_order_mu;
std::vector<std::unique_ptr<OrderEntry>> g_orders;

OrderEntry *order_entry_locked(const BtreeStream &S) {
    for (auto &e : g_orders)
        if (e->n == S.g.n && e->b == S.g.b && e->tile_keys == S.tile_keys) return e.get();
    if (g_orders.size() >= kMaxOrderEntries) return nullptr;
    auto e = std::make_unique<OrderEntry>();
    e->n = S.g.n;
    e->b = S.g.b;
    e->tile_keys = S.tile_keys;
    btree_compute_order(S, e->v);
    g_orders.push_back(std::move(e));
    return g_orders.back().get();
}
}  // namespace

bool btree_order_prepare(const BtreeStream &S, cudaStream_t st) {
    {
        std::lock_guard<std::mutex> lk(g_order_mu);
        for (auto &e : g_orders)
            if (e->n == S.g.n && e->b == S.g.b && e->tile_keys == S.tile_keys) return true;
        if (g_orders.size() >= kMaxOrderEntries) return false;
    }
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(st, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) {
        cudaGetLastError();
        return false;
    }
    auto e = std::make_unique<OrderEntry>();
    e->n = S.g.n;
    e->b = S.g.b;
    e->tile_keys = S.tile_keys;
    if (!btree_compute_order_device(S, st, e->v)) return false;
    std::lock_guard<std::mutex> lk(g_order_mu);
    for (auto &x : g_orders)
        if (x->n == S.g.n && x->b == S.g.b && x->tile_keys == S.tile_keys) return true;  // another thread's
    if (g_orders.size() >= kMaxOrderEntries) return false;
    g_orders.push_back(std::move(e));
    return true;
}

bool btree_order_host(const BtreeStream &S, OrderTables &t) {
    std::lock_guard<std::mutex> lk(g_order_mu);
    OrderEntry *e = order_entry_locked(S);
    if (!e) return false;
    t = e->v.tables();
    return true;
}

bool btree_order_device(const BtreeStream &S, cudaStream_t st, OrderTables &t) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxOrderDevices) return false;
    std::lock_guard<std::mutex> lk(g_order_mu);
    OrderEntry *e = order_entry_locked(S);
    if (!e) return false;
    const uint64_t N = S.ntiles, L = e->v.segs.size();
    if (!e->dev[dev]) {
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        if (cudaStreamIsCapturing(st, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) return false;
        char *p = nullptr;
        const size_t o1 = L * sizeof(FixSeg), o2 = o1 + N * sizeof(uint2);
        if (cudaMalloc(reinterpret_cast<void **>(&p), o2 + N * sizeof(uint32_t)) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        // copies on st, then a wait for them: a plain cudaMemcpy from pageable
        // memory may return before its DMA lands, and a non-blocking stream
        // would not wait for it
        if ((L && cudaMemcpyAsync(p, e->v.segs.data(), o1, cudaMemcpyHostToDevice, st) != cudaSuccess) ||
            cudaMemcpyAsync(p + o1, e->v.tab.data(), N * sizeof(uint2), cudaMemcpyHostToDevice, st) != cudaSuccess ||
            cudaMemcpyAsync(p + o2, e->v.order.data(), N * sizeof(uint32_t), cudaMemcpyHostToDevice, st) !=
                cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess) {
            cudaGetLastError();
            cudaFree(p);
            return false;
        }
        e->dev[dev] = p;
    }
    const char *p = static_cast<const char *>(e->dev[dev]);
    t.segs = reinterpret_cast<const FixSeg *>(p);
    t.nsegs = L;
    t.tab = reinterpret_cast<const uint2 *>(p + L * sizeof(FixSeg));
    t.order = reinterpret_cast<const uint32_t *>(p + L * sizeof(FixSeg) + N * sizeof(uint2));
    t.ranges = e->v.ranges.data();
    t.nranges = e->v.ranges.size();
    t.scratch_tiles = e->v.scratch_tiles;
    return true;
}

}  // namespace tl
