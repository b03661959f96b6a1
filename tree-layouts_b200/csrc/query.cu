// Batched exact point queries over the three layouts (sm_100a).
//
// Each kernel is persistent (grid = SMs x resident CTAs) and walks the query
// array with a grid stride.  The first P positions of the layout - the top
// levels for every layout, since each one stores its root region first - are
// copied once per CTA into shared memory, so the first levels of every descent
// cost a shared-memory load instead of an L2/HBM round trip.
//
// Answers are the layout position of the key or n (gpu/src/query-bst.cuh:41,
// gpu/src/query-btree.cuh:59, gpu/src/query-mveb.cuh:65).  For keys present in
// the layout the descent visits the same nodes as the reference's searches.
#include <algorithm>

#include "internal.h"
#include "tl_common.cuh"

namespace tl {

constexpr int kQueryThreads = 256;
constexpr uint32_t kPinBytes = 48 * 1024;
// A grouped batch over a BST of 256 MB or more pins fewer top levels, leaving
// room for 8 blocks an SM: measured on B200, 2^27 grouped queries, 2^30 - 1 u64
// keys 13.25 -> 12.14 ms, 2^27 - 1 u32 10.23 -> 9.79 ms (8 KB: the same); over
// a 128 MB tree 11.0 -> 11.6 ms, so not there
constexpr uint32_t kBstGroupPinBytes = 16 * 1024;

template <typename K>
__device__ __forceinline__ void pin_prefix(const K *__restrict__ A, uint64_t P, K *sm) {
    for (uint64_t x = threadIdx.x; x < P; x += blockDim.x) sm[x] = __ldg(A + x);
    __syncthreads();
}

template <typename K>
__device__ __forceinline__ K key_at(const K *__restrict__ A, const K *sm, uint64_t P, uint64_t i) {
    return i < P ? sm[i] : __ldg(A + i);
}

// ---------------------------------------------------------------- BST
// searchBST (gpu/src/query-bst.cuh:31-42): i = 2i + 1 + (q > A[i]).
template <typename K>
__global__ void __launch_bounds__(kQueryThreads)
bst_query_kernel(const K *__restrict__ A, uint64_t n, uint64_t P, const K *__restrict__ Q, uint64_t nq,
                 const uint32_t *__restrict__ perm, uint64_t *__restrict__ ans) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    K *sm = reinterpret_cast<K *>(smem_raw);
    pin_prefix(A, P, sm);
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t qi = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; qi < nq; qi += stride) {
        const K q = __ldcs(Q + qi);
        uint64_t i = 0, res = n;
        while (i < n) {
            const K cur = key_at(A, sm, P, i);
            if (q == cur) {
                res = i;
                break;
            }
            i = 2 * i + 1 + (q > cur);
        }
        const uint64_t out = perm ? (uint64_t)__ldg(perm + qi) : qi;
        if (out < nq) __stcs(ans + out, res);
    }
}

// ---------------------------------------------------------------- sorted array
// The binary-search comparator (gpu/src/binary-search.cuh:27-57 searches the
// sorted array before any permutation).  Branch-free lower bound: with
// len_0 = n and base_0 = 0, step d probes base_d + half_d (half_d = len_d / 2),
// base_{d+1} = base_d + half_d when that key is below the query, len_{d+1} =
// len_d - half_d; then the answer is the lower bound if it holds the query,
// else n.  The lengths do not depend on the query, so the keys probed in the
// first L steps form a complete binary tree of 2^L - 1 positions; they are
// pinned in shared memory in breadth-first order (node i has children 2i and
// 2i + 1, path bit = "went right"), which turns those steps into
// shared-memory loads.
template <typename K>
__global__ void __launch_bounds__(kQueryThreads)
sorted_query_kernel(const K *__restrict__ A, uint64_t n, uint32_t L, const K *__restrict__ Q, uint64_t nq,
                    uint64_t *__restrict__ ans) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    K *tree = reinterpret_cast<K *>(smem_raw);  // tree[1 .. 2^L - 1]
    const uint32_t nodes = (1u << L) - 1;
    for (uint32_t node = threadIdx.x + 1; node <= nodes; node += blockDim.x) {
        // replay the path of `node`: its bits below the leading one, high to low
        const uint32_t depth = 31 - __clz(node);
        uint64_t base = 0, len = n;
        for (uint32_t d = 0; d < depth; ++d) {
            const uint64_t half = len >> 1;
            if ((node >> (depth - 1 - d)) & 1u) base += half;
            len -= half;
        }
        tree[node] = __ldg(A + base + (len >> 1));
    }
    __syncthreads();
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t qi = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; qi < nq; qi += stride) {
        const K q = __ldcs(Q + qi);
        uint64_t base = 0, len = n;
        uint32_t node = 1;
        for (uint32_t d = 0; d < L; ++d) {  // len > 1 throughout: L < log2(n)
            const uint64_t half = len >> 1;
            const bool right = tree[node] < q;
            base += right ? half : 0;
            len -= half;
            node = 2 * node + right;
        }
        while (len > 1) {
            const uint64_t half = len >> 1;
            base += __ldg(A + base + half) < q ? half : 0;
            len -= half;
        }
        const K at = __ldg(A + base);
        const uint64_t lb = base + (at < q);
        __stcs(ans + qi, (lb < n && (lb == base ? at : __ldg(A + lb)) == q) ? lb : n);
    }
}

// ---------------------------------------------------------------- B-tree
// searchBtree (cpu/src/query-btree.h:33-54): the child followed is the number of
// node keys smaller than the query; an equal key ends the search.  A group of G
// lanes reads one node cooperatively: lane j of the group owns node slots
// j, j+G, ...; slots at or past n (the partial last leaf) count as +infinity.
template <typename K, int G>
__global__ void __launch_bounds__(kQueryThreads)
btree_query_kernel(const K *__restrict__ A, uint64_t n, uint64_t b, uint64_t P, const K *__restrict__ Q,
                   uint64_t nq, uint64_t *__restrict__ ans) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    K *sm = reinterpret_cast<K *>(smem_raw);
    pin_prefix(A, P, sm);
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t gl = lane % G;                      // lane within the group
    const uint32_t gbase = lane - gl;                  // first lane of the group
    const unsigned gmask = (G == 32 ? 0xFFFFFFFFu : ((1u << G) - 1)) << gbase;
    const uint64_t groups = (uint64_t)gridDim.x * blockDim.x / G;
    const uint64_t gid = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) / G;
    const uint64_t rounds = (nq + groups - 1) / groups;  // uniform trip count keeps warps converged
    for (uint64_t rd = 0; rd < rounds; ++rd) {
        const uint64_t qi = rd * groups + gid;
        const bool active = qi < nq;
        const K q = active ? Q[qi] : K(0);
        uint64_t i = 0, res = n;
        bool done = !active;
        while (__any_sync(0xFFFFFFFFu, !done)) {
            if (!done && i >= n) done = true;
            uint32_t lt = 0;
            int eq_slot = -1;
            if (!done) {
                for (uint64_t s = gl; s < b; s += G) {
                    const uint64_t p = i + s;
                    if (p < n) {
                        const K cur = key_at(A, sm, P, p);
                        lt += cur < q;
                        if (cur == q && eq_slot < 0) eq_slot = (int)s;
                    }
                }
            }
            // group reductions (all 32 lanes take part; inactive lanes add zero)
            for (int off = G / 2; off > 0; off >>= 1) {
                lt += __shfl_xor_sync(0xFFFFFFFFu, lt, off);
                const int o = __shfl_xor_sync(0xFFFFFFFFu, eq_slot, off);
                if (o >= 0 && (eq_slot < 0 || o < eq_slot)) eq_slot = o;
            }
            (void)gmask;
            if (!done) {
                // The reference returns the first equal key of the node whose
                // preceding keys are all smaller; with sorted nodes that is the
                // equal key at slot lt.
                if (eq_slot >= 0 && (uint64_t)eq_slot == lt) {
                    res = i + (uint64_t)eq_slot;
                    done = true;
                } else if (i + 1 > (n + 1) / (b + 1)) {
                    done = true;  // every child starts past n; also keeps (i+1)(b+1) from overflowing
                } else {
                    i = (i + 1) * (b + 1) + lt * b - 1;
                }
            }
        }
        if (active && gl == 0) ans[qi] = res;
    }
}

// One thread per query, for nodes of b*w = 16*NV bytes (node starts are then
// 16-byte aligned): the node is fetched with NV independent 16-byte loads.
template <typename K, int NV>
__global__ void __launch_bounds__(kQueryThreads)
btree_query_vec_kernel(const K *__restrict__ A, uint64_t n, uint64_t b, const K *__restrict__ Q, uint64_t nq,
                       uint64_t *__restrict__ ans) {
    constexpr int KPV = 16 / sizeof(K);  // keys per 16-byte vector
    constexpr int B = NV * KPV;          // == b
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t cmax = (n + 1) / (B + 1);
    for (uint64_t qi = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; qi < nq; qi += stride) {
        const K q = __ldcs(Q + qi);
        uint64_t i = 0, res = n;
        while (i < n) {
            uint32_t lt = 0;
            bool eq = false;
            if (i + B <= n) {
                const uint4 *node = reinterpret_cast<const uint4 *>(A + i);
                uint4 v[NV];
#pragma unroll
                for (int j = 0; j < NV; ++j) v[j] = __ldg(node + j);
#pragma unroll
                for (int j = 0; j < NV; ++j) {
                    const K *kk = reinterpret_cast<const K *>(&v[j]);
#pragma unroll
                    for (int e = 0; e < KPV; ++e) lt += kk[e] < q;
                }
                if (lt < (uint32_t)B) {
                    const K *all = reinterpret_cast<const K *>(v);
                    K at = all[0];
#pragma unroll
                    for (int j = 1; j < B; ++j)
                        if ((uint32_t)j == lt) at = all[j];
                    eq = at == q;
                }
            } else {
                const uint64_t valid = n - i;
                for (uint64_t j = 0; j < valid; ++j) lt += __ldg(A + i + j) < q;
                if (lt < valid) eq = __ldg(A + i + lt) == q;
            }
            if (eq) {
                res = i + lt;
                break;
            }
            if (i + 1 > cmax) break;
            i = (i + 1) * (B + 1) + (uint64_t)lt * B - 1;
        }
        __stcs(ans + qi, res);
    }
}

// One thread per query for nodes of NB = b * w bytes, NB a multiple of 32 on a
// 32-byte aligned layout: a node is NB / 32 independent 32-byte loads (one L1
// wavefront each when the warp's nodes are distinct lines, half the 16-byte
// loads' count).  The first P keys (whole top levels) may be pinned in shared
// memory.  The partial last leaf is read with guarded scalar loads.
template <typename K, int NB, bool kPin>
__global__ void __launch_bounds__(kQueryThreads)
btree_query_v32_kernel(const K *__restrict__ A, uint64_t n, uint64_t P, const K *__restrict__ Q, uint64_t nq,
                       uint64_t *__restrict__ ans) {
    constexpr int KPL = 32 / sizeof(K);  // keys per 32-byte load
    constexpr int NL = NB / 32;          // loads per node
    constexpr int B = NB / sizeof(K);    // == b
    extern __shared__ __align__(16) unsigned char smem_raw[];
    K *sm = reinterpret_cast<K *>(smem_raw);
    if constexpr (kPin) pin_prefix(A, P, sm);
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t cmax = (n + 1) / (B + 1);
    for (uint64_t qi = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; qi < nq; qi += stride) {
        const K q = __ldcs(Q + qi);
        uint64_t i = 0, res = n;
        while (i < n) {
            uint32_t lt = 0;
            bool eq = false;
            if (i + B <= n) {
                K v[NL][KPL];
                if (kPin && i < P) {
#pragma unroll
                    for (int j = 0; j < NL; ++j) {
                        const uint4 *s4 = reinterpret_cast<const uint4 *>(sm + i + j * KPL);
                        const uint4 a = s4[0], c = s4[1];
                        const K *ka = reinterpret_cast<const K *>(&a);
                        const K *kc = reinterpret_cast<const K *>(&c);
#pragma unroll
                        for (int e = 0; e < KPL / 2; ++e) {
                            v[j][e] = ka[e];
                            v[j][KPL / 2 + e] = kc[e];
                        }
                    }
                } else {
#pragma unroll
                    for (int j = 0; j < NL; ++j) ldg32(A + i + j * KPL, v[j]);
                }
#pragma unroll
                for (int j = 0; j < NL; ++j)
#pragma unroll
                    for (int e = 0; e < KPL; ++e) lt += v[j][e] < q;
#pragma unroll
                for (int j = 0; j < NL; ++j)
#pragma unroll
                    for (int e = 0; e < KPL; ++e) eq |= v[j][e] == q;
            } else {
                const uint64_t valid = n - i;
                for (uint64_t j = 0; j < valid; ++j) {
                    const K cur = __ldg(A + i + j);
                    lt += cur < q;
                    eq |= cur == q;
                }
            }
            if (eq) {
                res = i + lt;
                break;
            }
            if (i + 1 > cmax) break;
            i = (i + 1) * (B + 1) + (uint64_t)lt * B - 1;
        }
        __stcs(ans + qi, res);
    }
}

// G lanes per query read a node together with NL = NB / (32 G) 32-byte loads
// each (lane g holds slots g * KPL + j * G * KPL + [0, KPL) for load j).  Each
// load instruction of a warp then touches 32 / G node lines with G sectors of
// a line in one L1 wavefront, where a thread per query spends a wavefront per
// sector; fewer lanes per node keep more descents in flight.  Control flow is
// warp-uniform (a warp takes 32 / G queries per round and descends while any of
// them is live), so the group's count is a full-warp shuffle sum and an equal
// key in any of its lanes, found by ballot, ends its descent.  (Descending to
// the last level on counts alone and checking q's successor with one load at
// the end measured 9 % slower on B200: that load adds a dependent step to every
// warp's round.)
template <typename K, int NB, int G>
__global__ void __launch_bounds__(kQueryThreads)
btree_query_group32_kernel(const K *__restrict__ A, uint64_t n, const K *__restrict__ Q, uint64_t nq,
                           uint64_t *__restrict__ ans) {
    constexpr int KPL = 32 / sizeof(K);  // keys per 32-byte load
    constexpr int NL = NB / 32 / G;      // 32-byte loads per lane and node
    constexpr int B = NB / sizeof(K);    // == b
    constexpr int QPW = 32 / G;          // queries per warp and round
    static_assert(G >= 2 && G <= 8 && (G & (G - 1)) == 0 && NL >= 1 && NL * G * 32 == NB,
                  "group of 2, 4 or 8 lanes");
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t g = lane % G;
    const uint32_t gshift = lane - g;
    const uint64_t warps = (uint64_t)gridDim.x * (blockDim.x / 32);
    const uint64_t wid = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) / 32;
    const uint64_t cmax = (n + 1) / (B + 1);
    for (uint64_t base = wid * QPW; base < nq; base += warps * QPW) {
        const uint64_t qi = base + lane / G;
        bool live = qi < nq && n > 0;
        const K q = qi < nq ? __ldcs(Q + qi) : K(0);
        uint64_t i = 0, res = n;
        while (__any_sync(0xFFFFFFFFu, live)) {
            uint32_t lt = 0;
            bool eq = false;
            if (live) {
                const uint64_t s0 = i + (uint64_t)g * KPL;  // lane g: slots s0 + j * G * KPL + e
                if (i + B <= n) {
                    K v[NL][KPL];
#pragma unroll
                    for (int j = 0; j < NL; ++j) ldg32(A + s0 + (uint64_t)j * G * KPL, v[j]);
#pragma unroll
                    for (int j = 0; j < NL; ++j)
#pragma unroll
                        for (int e = 0; e < KPL; ++e) {
                            lt += v[j][e] < q;
                            eq |= v[j][e] == q;
                        }
                } else {  // the partial last leaf: slots at or past n do not count
#pragma unroll
                    for (int j = 0; j < NL; ++j)
#pragma unroll
                        for (int e = 0; e < KPL; ++e) {
                            const uint64_t p = s0 + (uint64_t)j * G * KPL + e;
                            if (p < n) {
                                const K cur = __ldg(A + p);
                                lt += cur < q;
                                eq |= cur == q;
                            }
                        }
                }
            }
#pragma unroll
            for (int off = G / 2; off > 0; off >>= 1) lt += __shfl_xor_sync(0xFFFFFFFFu, lt, off);
            const bool hit = ((__ballot_sync(0xFFFFFFFFu, eq) >> gshift) & ((1u << G) - 1)) != 0;
            if (live) {
                if (hit) {
                    res = i + lt;
                    live = false;
                } else if (i + 1 > cmax) {
                    live = false;
                } else {
                    i = (i + 1) * (B + 1) + (uint64_t)lt * B - 1;
                    live = i < n;
                }
            }
        }
        if (g == 0 && qi < nq) __stcs(ans + qi, res);
    }
}

static int g_query_variant = 0;
void set_query_variant(int v) { g_query_variant = v; }
int query_variant() { return g_query_variant; }

// ---------------------------------------------------------------- mvEB
// searchvEB (gpu/src/query-mveb.cuh:43-66): BFS index i and the table recurrence
// pos[d] = pos[D_d] + R_d + (i & R_d) * L_d, with pos[] in shared memory, one
// column per thread (32-bit entries when n < 2^32).  Tables are read through the
// read-only cache.  A descent past the deepest level ends as "absent" (the
// reference reads past its table there; it only ever issues hits).
constexpr int kVebThreads = 128;
constexpr size_t kVebMinPin = 8 * 1024;
// A batch grouped by value: neighbouring descents share most deep nodes (L1
// and L2 hits), so more of them in flight pays where it costs L1 hits on a
// batch as given.  Measured on B200, 2^27 grouped queries over 2^30 - 1 u32
// mvEB keys (grouping included): 128 threads and 48 KB a block 20.6 ms,
// 128 / 24 KB 15.0, 128 / 32 KB 17.7, 256 / 40 KB 14.3, 256 / 48 KB 14.0,
// 256 / 64 KB 16.0, 384 / 56 KB 13.6, 512 / 72 KB 13.5, 1024 / 136 KB
// 14.7 ms; shapes with more threads on the batch as given 46.6 to 56.4 ms
// against 40.0 (128 / 48 KB).
constexpr int kVebGroupThreads = 512;
constexpr size_t kVebGroupBudget = 72 * 1024;

// QK descents per thread in lock-step: every step takes all of a thread's
// unresolved queries one level down, so their key loads are in flight together
// and each level's table entry is read once for all of them.  A query leaves
// the step loop when it finds its key (res), falls off the tree (bit in
// `fell`: absent) or leaves the division [offset, limit) (neither: the caller
// tries the next division).  pos[] holds QK columns per thread:
// pos[(cd * QK + k) * T + tid].
template <typename K, typename PosT, int QK>
__device__ __forceinline__ void veb_descend_multi(const K *__restrict__ A, const K *sm, uint64_t P,
                                                  const tl_veb_table *__restrict__ tab, uint32_t d, const K (&q)[QK],
                                                  uint64_t offset, uint64_t limit, PosT *pos, uint32_t todo,
                                                  uint64_t (&res)[QK], uint32_t &fell) {
    const uint32_t T = blockDim.x, tid = threadIdx.x;
    uint64_t i[QK], index[QK];
#pragma unroll
    for (int k = 0; k < QK; ++k) {
        i[k] = 1;
        index[k] = 0;
        pos[k * T + tid] = 1;
    }
    uint32_t act = todo;
    uint32_t cd = 0;
    while (act) {
        K cur[QK];
#pragma unroll
        for (int k = 0; k < QK; ++k) {
            cur[k] = K(0);
            if ((act >> k) & 1u) {
                if (index[k] + offset < limit)
                    cur[k] = key_at(A, sm, P, offset + index[k]);
                else
                    act &= ~(1u << k);  // left the division: not resolved here
            }
        }
#pragma unroll
        for (int k = 0; k < QK; ++k)
            if (((act >> k) & 1u) && q[k] == cur[k]) {
                res[k] = offset + index[k];
                act &= ~(1u << k);
            }
        if (!act) break;
        if (cd + 1 >= d) {
            fell |= act;
            break;
        }
        ++cd;
        const uint64_t L = __ldg(&tab[cd].L), R = __ldg(&tab[cd].R);
        const uint32_t D = __ldg(&tab[cd].D);
        if (D >= cd) {  // not a table built by buildTable: stop instead of reading outside pos[]
            fell |= act;
            break;
        }
#pragma unroll
        for (int k = 0; k < QK; ++k)
            if ((act >> k) & 1u) {
                i[k] = 2 * i[k] + (q[k] > cur[k]);
                const uint64_t p = (uint64_t)pos[(D * QK + k) * T + tid] + R + (i[k] & R) * L;
                pos[(cd * QK + k) * T + tid] = (PosT)p;
                index[k] = p - 1;
            }
    }
}

// idx == nullptr: perfect layout, one table (timeQueryvEB); otherwise the
// non-perfect table set (timeQueryvEB_nonperfect): the divisions in order, each
// query until it is resolved.  A block takes QK * T consecutive queries at a
// time, thread t the queries t, t + T, ...
template <typename K, typename PosT, int QK, int kThreads>
__global__ void __launch_bounds__(kThreads)
veb_query_kernel(const K *__restrict__ A, uint64_t n, uint64_t P, uint32_t dmax,
                 const tl_veb_table *__restrict__ tables, const uint64_t *__restrict__ idx,
                 const uint32_t *__restrict__ table_idx, uint32_t num_tables, const K *__restrict__ Q,
                 uint64_t nq, const uint32_t *__restrict__ perm, uint64_t *__restrict__ ans) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    PosT *pos = reinterpret_cast<PosT *>(smem_raw);
    K *sm = reinterpret_cast<K *>(smem_raw + ((size_t)dmax * QK * blockDim.x * sizeof(PosT) + 15) / 16 * 16);
    pin_prefix(A, P, sm);
    const uint64_t T = blockDim.x;
    for (uint64_t base = (uint64_t)blockIdx.x * QK * T; base < nq; base += (uint64_t)gridDim.x * QK * T) {
        K q[QK];
        uint64_t res[QK];
        uint32_t todo = 0, fell = 0;
#pragma unroll
        for (int k = 0; k < QK; ++k) {
            const uint64_t qi = base + k * T + threadIdx.x;
            res[k] = n;
            q[k] = K(0);
            if (qi < nq) {
                q[k] = __ldcs(Q + qi);
                todo |= 1u << k;
            }
        }
        if (!idx) {
            veb_descend_multi<K, PosT, QK>(A, sm, P, tables, bit_length(n), q, 0, n, pos, todo, res, fell);
        } else {
            uint64_t offset = 0;
            for (uint32_t j = 0; j < num_tables && todo; ++j) {
                const uint64_t lim = __ldg(idx + j);
                veb_descend_multi<K, PosT, QK>(A, sm, P, tables + __ldg(table_idx + j), bit_length(n - offset), q,
                                               offset, lim, pos, todo, res, fell);
#pragma unroll
                for (int k = 0; k < QK; ++k)
                    if (res[k] != n) todo &= ~(1u << k);  // found
                todo &= ~fell;                             // absent
                offset = lim;
            }
        }
#pragma unroll
        for (int k = 0; k < QK; ++k) {
            const uint64_t qi = base + k * T + threadIdx.x;
            const uint64_t out = qi < nq ? (perm ? (uint64_t)__ldg(perm + qi) : qi) : nq;
            if (out < nq) __stcs(ans + out, res[k]);
        }
    }
}

// ---------------------------------------------------------------- partition
// Queries close in value walk close paths through a BST or vEB layout, whose
// lower levels hold each subtree's keys together.  Grouping a batch by value
// lets a node fetched once from HBM serve the rest of its group from L2 or L1.
// The batch is split into 2^bits buckets of its value range [min q, max q]
// (bucket = (q - min q) >> shift, shift fitting the range to `bits` bits) by
// bits / 4 passes over 4 bits each, most significant first; `bits` grows with
// the batch (part_bits) up to 20.  A pass gives every block
// tiles of kPartTile entries; within each segment of the previous pass that a
// tile touches it ranks the entries into 16 bins in shared memory, reserves
// one global range per (segment, bin) with a single atomic, and writes each
// bin's entries out as one contiguous run.  The same pass counts the entries
// of every (segment, bin) by the next digit, so only the first pass needs a
// counting sweep of its own.  Order within a bucket is not kept (the search
// does not need it).  The search kernels write each answer through the
// carried index, so the answers keep the batch's order.
constexpr uint32_t kPartMaxBits = 20, kPartBuckets = 1u << kPartMaxBits;
constexpr uint32_t kPartDigit = 4, kPartBins = 1u << kPartDigit;
// Entries a segment of the last pass holds on average, at least: a tile that
// meets many small segments takes one portion at a time (measured on B200,
// 2^20 queries into 2^20 buckets: the last pass 0.61 ms, the whole search
// 0.06 ms; 2048 measured as fast as 1024 or faster from 2^20 to 2^27 queries)
constexpr uint64_t kPartMinSegment = 2048;
constexpr int kPartThreads = 256;
constexpr uint32_t kPartScanChunk = 4096;  // counts scanned by one block of 1024 threads
static_assert(kPartBins * kPartBins == kPartThreads, "one next-digit counter per thread");
static_assert(kPartBuckets / kPartScanChunk <= 1024, "chunk totals fit one block");
// entries per tile: the staging area of values, indices and bins in under 48 KB
template <typename K>
constexpr uint32_t part_tile() {
    return sizeof(K) == 8 ? 3584 : 4096;
}

template <typename K>
__global__ void qpart_minmax_kernel(const K *__restrict__ Q, uint64_t q, unsigned long long *__restrict__ mm) {
    unsigned long long lo = ~0ull, hi = 0;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < q; i += (uint64_t)gridDim.x * blockDim.x) {
        const unsigned long long v = (unsigned long long)Q[i];
        lo = v < lo ? v : lo;
        hi = v > hi ? v : hi;
    }
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long a = __shfl_xor_sync(0xFFFFFFFFu, lo, o), b = __shfl_xor_sync(0xFFFFFFFFu, hi, o);
        lo = a < lo ? a : lo;
        hi = b > hi ? b : hi;
    }
    __shared__ unsigned long long s_lo[32], s_hi[32];  // one atomic pair per block, not per warp
    if ((threadIdx.x & 31) == 0) {
        s_lo[threadIdx.x >> 5] = lo;
        s_hi[threadIdx.x >> 5] = hi;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (uint32_t w = 1; w < blockDim.x / 32; ++w) {
            lo = s_lo[w] < lo ? s_lo[w] : lo;
            hi = s_hi[w] > hi ? s_hi[w] : hi;
        }
        atomicMin(&mm[0], lo);
        atomicMax(&mm[1], hi);
    }
}

// The bucket of value v is the `bits` bits of (v - min q) below the top of
// the range [min q, max q]: (v - min q) >> qpart_bucket_shift(mm, bits)
__device__ __forceinline__ uint32_t qpart_bucket_shift(const unsigned long long *mm, uint32_t bits) {
    const uint32_t span = bit_length((uint64_t)(mm[1] - mm[0]));
    return span > bits ? span - bits : 0;
}

// The first segment s in [lo, nseg) whose end seg_end[s] is above a, found by
// one warp: each round probes 32 ends spread over the open range.  Needs
// seg_end non-decreasing, seg_end[s] <= a for s < lo and seg_end[nseg - 1] > a.
// consecutive: probe lo .. lo + 31 first (a portion that ended at a segment's
// end is usually followed by the next segment).
__device__ __forceinline__ uint32_t qpart_find_segment(const uint32_t *__restrict__ seg_end, uint32_t lo,
                                                       uint32_t nseg, uint64_t a, bool consecutive) {
    const uint32_t lane = threadIdx.x & 31;
    uint32_t hi = nseg;
    uint32_t step = consecutive ? 1 : (hi - lo + 31) / 32;
    for (;;) {
        const uint32_t at = min(lo + (lane + 1) * step - 1, hi - 1);
        const uint32_t hit = __ballot_sync(0xFFFFFFFFu, seg_end[at] > a);
        if (hit == 0) {  // all 32 probes at or below a (only in a consecutive round below hi)
            lo += 32 * step;
            step = (hi - lo + 31) / 32;
            continue;
        }
        const uint32_t f = __ffs(hit) - 1;
        const uint32_t at_f = min(lo + (f + 1) * step - 1, hi - 1);
        if (step == 1) return at_f;
        lo += f * step;  // just past the probe before the first hit
        hi = at_f + 1;
        step = (hi - lo + 31) / 32;
    }
}

// One pass (pass p takes bucket bits [bits - 4(p+1), bits - 4p))
// over entries [0, q) of (vals, idx) (idx == nullptr: the entry's own index).
// seg_end[0 .. nseg) are the exclusive ends of the previous pass's segments
// (nseg = 16^p; pass 0: one segment).  mode 0 adds the tiles' bin counts to
// count[seg * 16 + bin]; mode 1 scatters through cursor[] (count[] scanned)
// into (ovals, oidx) and, with next != nullptr, adds the counts of the next
// digit to next[(seg * 16 + bin) * 16 + next digit].
template <typename K>
__global__ void __launch_bounds__(kPartThreads)
qpart_pass_kernel(int mode, uint32_t bits, uint32_t pass, const K *__restrict__ vals, const uint32_t *__restrict__ idx, uint64_t q,
                  const unsigned long long *__restrict__ mm, const uint32_t *__restrict__ seg_end, uint32_t nseg,
                  uint32_t *__restrict__ count, K *__restrict__ ovals, uint32_t *__restrict__ oidx,
                  uint32_t *__restrict__ next) {
    constexpr uint32_t kPartTile = part_tile<K>();
    constexpr int kItems = kPartTile / kPartThreads;
    __shared__ K sv[kPartTile];
    __shared__ uint32_t si[kPartTile];
    __shared__ uint8_t sb[kPartTile];  // the bin of each staged entry
    __shared__ uint32_t cnt[kPartBins], off[kPartBins], run[kPartBins], base[kPartBins];
    __shared__ uint32_t nxt[kPartBins * kPartBins];
    __shared__ uint32_t s_seg[2];
    const uint64_t qmin = mm[0];
    const uint32_t shift = qpart_bucket_shift(mm, bits) + bits - kPartDigit * (pass + 1);  // this digit
    const bool count_next = mode == 1 && next != nullptr && pass + 1 < bits / kPartDigit;
    for (uint64_t t0 = (uint64_t)blockIdx.x * kPartTile; t0 < q; t0 += (uint64_t)gridDim.x * kPartTile) {
        const uint64_t t1 = min(q, t0 + kPartTile);
        uint64_t a = t0;
        uint32_t seg = 0;
        while (a < t1) {  // one segment of the previous pass at a time
            __syncthreads();
            if (threadIdx.x < 32) {  // the segment holding entry a
                const uint32_t s =
                    nseg > 1 ? qpart_find_segment(seg_end, a == t0 ? 0 : seg + 1, nseg, a, a != t0) : 0;
                if (threadIdx.x == 0) {
                    s_seg[0] = s;
                    s_seg[1] = nseg > 1 ? seg_end[s] : (uint32_t)q;  // pass 0: one segment [0, q)
                }
            }
            if (threadIdx.x < kPartBins) {
                cnt[threadIdx.x] = 0;
                run[threadIdx.x] = 0;
            }
            nxt[threadIdx.x] = 0;
            __syncthreads();
            seg = s_seg[0];
            uint64_t b = min(t1, (uint64_t)s_seg[1]);
            if (b <= a) b = t1;  // cannot happen (the last end is q); both modes take the same steps
            const uint32_t len = (uint32_t)(b - a);
            // this thread's entries j = threadIdx.x + i * kPartThreads of the
            // portion, values and indices loaded together (their latencies
            // overlap) and kept in registers
            K v[kItems];
            uint32_t id[kItems];
#pragma unroll
            for (int i = 0; i < kItems; ++i) {
                const uint32_t j = threadIdx.x + i * kPartThreads;
                v[i] = j < len ? vals[a + j] : K(0);
                id[i] = mode == 1 && idx && j < len ? idx[a + j] : (uint32_t)(a + j);
            }
#pragma unroll
            for (int i = 0; i < kItems; ++i) {
                const uint32_t j = threadIdx.x + i * kPartThreads;
                if (j < len) atomicAdd(&cnt[(((uint64_t)v[i] - qmin) >> shift) & (kPartBins - 1)], 1u);
            }
            __syncthreads();
            if (mode == 0) {
                if (threadIdx.x < kPartBins && cnt[threadIdx.x])
                    atomicAdd(&count[seg * kPartBins + threadIdx.x], cnt[threadIdx.x]);
            } else {
                if (threadIdx.x == 0) {
                    uint32_t o = 0;
                    for (uint32_t k = 0; k < kPartBins; ++k) {
                        off[k] = o;
                        o += cnt[k];
                    }
                }
                if (threadIdx.x < kPartBins && cnt[threadIdx.x])
                    base[threadIdx.x] = atomicAdd(&count[seg * kPartBins + threadIdx.x], cnt[threadIdx.x]);
                __syncthreads();
#pragma unroll
                for (int i = 0; i < kItems; ++i) {  // rank into the staging area
                    const uint32_t j = threadIdx.x + i * kPartThreads;
                    if (j < len) {
                        const uint64_t rel = (uint64_t)v[i] - qmin;
                        const uint32_t bin = (uint32_t)(rel >> shift) & (kPartBins - 1);
                        const uint32_t r = off[bin] + atomicAdd(&run[bin], 1u);
                        sv[r] = v[i];
                        si[r] = id[i];
                        sb[r] = (uint8_t)bin;
                        if (count_next)
                            atomicAdd(&nxt[bin * kPartBins +
                                           ((uint32_t)(rel >> (shift - kPartDigit)) & (kPartBins - 1))],
                                      1u);
                    }
                }
                if (threadIdx.x < kPartBins) base[threadIdx.x] -= off[threadIdx.x];  // bin's entry j goes to base + j
                __syncthreads();
                for (uint32_t j = threadIdx.x; j < len; j += blockDim.x) {  // each bin as one run
                    const uint32_t p = base[sb[j]] + j;
                    ovals[p] = sv[j];
                    oidx[p] = si[j];
                }
                // (segment, bin) of this pass is segment seg * 16 + bin of the
                // next: its counters start at (seg * 16 + bin) * 16
                if (count_next && nxt[threadIdx.x])
                    atomicAdd(&next[(uint64_t)seg * kPartBins * kPartBins + threadIdx.x], nxt[threadIdx.x]);
            }
            a = b;
        }
    }
}

// Exclusive scan of count[0, m) in place, m a multiple of kPartScanChunk: block
// c scans chunk c; ends (when given) gets the inclusive sums and total[c] the
// chunk's sum.  With more than one chunk, qpart_scan_add_kernel then adds the
// sums of the chunks before each one.
__global__ void __launch_bounds__(1024) qpart_scan_kernel(uint32_t *__restrict__ count, uint32_t *__restrict__ ends,
                                                          uint32_t *__restrict__ total) {
    static_assert(kPartScanChunk == 4 * 1024, "four counts a thread");
    __shared__ uint32_t wsum[32];
    const uint64_t at = (uint64_t)blockIdx.x * kPartScanChunk + threadIdx.x * 4;
    const uint4 c = *reinterpret_cast<const uint4 *>(count + at);
    const uint32_t sum = c.x + c.y + c.z + c.w;
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t inc = sum;  // inclusive scan within the warp
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xFFFFFFFFu, inc, o);
        if (lane >= (uint32_t)o) inc += t;
    }
    if (lane == 31) wsum[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = wsum[lane];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(0xFFFFFFFFu, w, o);
            if (lane >= (uint32_t)o) w += t;
        }
        wsum[lane] = w;  // inclusive over warps
        if (lane == 31 && total) total[blockIdx.x] = w;
    }
    __syncthreads();
    const uint32_t r0 = (warp ? wsum[warp - 1] : 0) + inc - sum;
    const uint4 ex = make_uint4(r0, r0 + c.x, r0 + c.x + c.y, r0 + c.x + c.y + c.z);
    *reinterpret_cast<uint4 *>(count + at) = ex;
    if (ends) *reinterpret_cast<uint4 *>(ends + at) = make_uint4(ex.y, ex.z, ex.w, ex.w + c.w);
}

// Block c of the grid adds the sums of chunks [0, c + 1) to chunk c + 1.
__global__ void __launch_bounds__(1024) qpart_scan_add_kernel(uint32_t *__restrict__ count,
                                                              uint32_t *__restrict__ ends,
                                                              const uint32_t *__restrict__ total) {
    __shared__ uint32_t s_off;
    const uint32_t chunk = blockIdx.x + 1;
    if (threadIdx.x < 32) {
        uint32_t o = 0;
        for (uint32_t k = threadIdx.x; k < chunk; k += 32) o += total[k];
        o = __reduce_add_sync(0xFFFFFFFFu, o);
        if (threadIdx.x == 0) s_off = o;
    }
    __syncthreads();
    const uint32_t o = s_off;
    const uint64_t at = (uint64_t)chunk * kPartScanChunk + threadIdx.x * 4;
    uint4 c = *reinterpret_cast<const uint4 *>(count + at);
    *reinterpret_cast<uint4 *>(count + at) = make_uint4(c.x + o, c.y + o, c.z + o, c.w + o);
    if (ends) {
        c = *reinterpret_cast<const uint4 *>(ends + at);
        *reinterpret_cast<uint4 *>(ends + at) = make_uint4(c.x + o, c.y + o, c.z + o, c.w + o);
    }
}

static int query_sm_count();

// Device memory of one partitioned batch: stream-ordered, freed (on the same
// stream, after the search kernel) when the launch function returns.
struct QueryPartition {
    void *buf = nullptr;
    const void *qs = nullptr;
    const uint32_t *perm = nullptr;
    cudaStream_t st = nullptr;
    ~QueryPartition() {
        if (buf) cudaFreeAsync(buf, st);
    }
};

// Bucket bits for a batch of q queries: the most (a multiple of 4, at most
// kPartMaxBits) whose last pass still has kPartMinSegment entries a segment
// on average, and at least 4.
static uint32_t part_bits(uint64_t q) {
    uint32_t bits = kPartDigit;
    while (bits + kPartDigit <= kPartMaxBits && (q >> bits) >= kPartMinSegment) bits += kPartDigit;
    return bits;
}

template <typename K>
static int partition_queries(const K *Q, uint64_t q, cudaStream_t st, QueryPartition &out) {
    auto al = [](uint64_t x) { return (x + 255) / 256 * 256; };
    auto padded = [](uint32_t m) { return (m + kPartScanChunk - 1) / kPartScanChunk * kPartScanChunk; };
    const uint32_t bits = part_bits(q), passes = bits / kPartDigit;
    // mm and the scan's chunk totals | the counts of this pass and of the
    // next (up to 2^bits each) | segment ends of the previous pass and of
    // this one | two (vals, idx) buffers
    const uint64_t b_mm = 256 + 4096, b_c = al(padded(1u << bits) * 4ull), b_v = al(q * sizeof(K)),
                   b_i = al(q * 4);
    char *buf = nullptr;
    keep_pool_memory();
    if (cudaMallocAsync(reinterpret_cast<void **>(&buf), b_mm + 4 * b_c + 2 * (b_v + b_i), st) != cudaSuccess) {
        cudaGetLastError();
        return TL_ERROR_OUT_OF_MEMORY;
    }
    out.buf = buf;  // freed by out's destructor on every path from here
    out.st = st;
    char *p = buf;
    unsigned long long *mm = reinterpret_cast<unsigned long long *>(p);
    uint32_t *total = reinterpret_cast<uint32_t *>(p + 256);
    p += b_mm;
    uint32_t *cnt[2] = {reinterpret_cast<uint32_t *>(p), reinterpret_cast<uint32_t *>(p + b_c)};
    p += 2 * b_c;
    uint32_t *ends[2] = {reinterpret_cast<uint32_t *>(p), reinterpret_cast<uint32_t *>(p + b_c)};
    p += 2 * b_c;
    K *v[2] = {reinterpret_cast<K *>(p), reinterpret_cast<K *>(p + b_v + b_i)};
    uint32_t *ix[2] = {reinterpret_cast<uint32_t *>(p + b_v), reinterpret_cast<uint32_t *>(p + 2 * b_v + b_i)};
    TL_CUDA_TRY(cudaMemsetAsync(mm, 0xFF, 8, st));  // min: all ones
    TL_CUDA_TRY(cudaMemsetAsync(mm + 1, 0, 8, st));
    const unsigned g = (unsigned)std::min<uint64_t>((q + 255) / 256, (uint64_t)query_sm_count() * 8);
    qpart_minmax_kernel<K><<<g, 256, 0, st>>>(Q, q, mm);
    const unsigned gt =
        (unsigned)std::min<uint64_t>((q + part_tile<K>() - 1) / part_tile<K>(), (uint64_t)query_sm_count() * 8);
    const K *src_v = Q;
    const uint32_t *src_i = nullptr;
    uint32_t nseg = 1;
    TL_CUDA_TRY(cudaMemsetAsync(cnt[0], 0, (size_t)padded(kPartBins) * 4, st));
    qpart_pass_kernel<K><<<gt, kPartThreads, 0, st>>>(0, bits, 0, src_v, src_i, q, mm, ends[1], 1, cnt[0], nullptr,
                                                      nullptr, nullptr);
    for (uint32_t pass = 0; pass < passes; ++pass) {
        const uint32_t m = nseg * kPartBins;  // this pass's buckets
        const uint32_t *seg = ends[(pass + 1) & 1];
        uint32_t *next_ends = ends[pass & 1];
        uint32_t *count = cnt[pass & 1], *next = nullptr;
        const uint32_t chunks = padded(m) / kPartScanChunk;
        qpart_scan_kernel<<<chunks, 1024, 0, st>>>(count, next_ends, total);
        if (chunks > 1) qpart_scan_add_kernel<<<chunks - 1, 1024, 0, st>>>(count, next_ends, total);
        if (pass + 1 < passes) {
            next = cnt[(pass + 1) & 1];
            TL_CUDA_TRY(cudaMemsetAsync(next, 0, (size_t)padded(m * kPartBins) * 4, st));
        }
        K *dv = v[pass & 1];
        uint32_t *di = ix[pass & 1];
        qpart_pass_kernel<K><<<gt, kPartThreads, 0, st>>>(1, bits, pass, src_v, src_i, q, mm, seg, nseg, count, dv,
                                                          di, next);
        src_v = dv;
        src_i = di;
        nseg = m;
    }
    TL_CUDA_TRY(cudaGetLastError());
    out.qs = src_v;
    out.perm = src_i;
    return TL_SUCCESS;
}

// ---------------------------------------------------------------- host
static int g_qsm = 0;
static int query_sm_count() {
    if (!g_qsm) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&g_qsm, cudaDevAttrMultiProcessorCount, dev);
        if (g_qsm <= 0) g_qsm = 148;
    }
    return g_qsm;
}

template <typename Kern>
static int persistent_grid(Kern kern, size_t smem, uint64_t work_threads, unsigned *grid) {
    TL_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    TL_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kQueryThreads, smem));
    uint64_t g = (uint64_t)std::max(per_sm, 1) * query_sm_count();
    uint64_t need = (work_threads + kQueryThreads - 1) / kQueryThreads;
    *grid = (unsigned)std::max<uint64_t>(1, std::min(g, need));
    return TL_SUCCESS;
}

template <typename K>
static int launch_query(const QueryArgs &a, cudaStream_t st) {
    const K *A = static_cast<const K *>(a.layout_keys);
    const K *Q = static_cast<const K *>(a.queries);
    uint64_t P = std::min<uint64_t>(a.n, kPinBytes / sizeof(K));
    unsigned grid = 1;
    // BST and vEB descents search a batch of 2^21 queries or more grouped by
    // value, over a vEB layout of 4 MB or more and a BST of 64 MB or more.
    // Measured on B200, as given against grouped (grouping included): mvEB
    // 2^30 - 1 u32, 2^27 queries 39.8 / 13.5 ms; mvEB 2^20 - 1 u32, 2^22
    // queries 0.49 / 0.32 ms, 2^20 queries 0.14 / 0.14; BST 2^23 - 1 u64 (64
    // MB), 2^22 queries 0.39 / 0.31 ms, 2^20 queries 0.11 / 0.13; BST 2^22 - 1
    // u64 (32 MB) 0.30 / 0.29 at 2^22 and 9.2 / 11.4 ms at 2^27 queries.
    // B-tree nodes gain little even sorted (9.45 against 8.28 ms) and keep the
    // batch's order.  Measurement hooks: variant 19 never groups, 20 always.
    QueryPartition part;
    const uint32_t *perm = nullptr;
    const uint64_t tree_bytes = a.n * sizeof(K);
    const bool large = a.layout == Q_BST ? tree_bytes >= (64ull << 20) : tree_bytes >= (4ull << 20);
    if ((a.layout == Q_BST || a.layout == Q_VEB || a.layout == Q_VEB_NP) && g_query_variant != 19 &&
        a.q < (1ull << 32) && (g_query_variant == 20 || (a.q >= (1ull << 21) && large))) {
        const int rc = partition_queries<K>(Q, a.q, st, part);
        if (rc == TL_SUCCESS) {
            Q = static_cast<const K *>(part.qs);
            perm = part.perm;
        } else if (rc != TL_ERROR_OUT_OF_MEMORY) {
            return rc;  // out of memory: the batch is searched as given
        }
    }
    if (a.layout == Q_SORTED) {
        // pinned probe tree: L levels with 2^L - 1 < n (so every pinned step has
        // len > 1) and at most 32 KB of keys
        uint32_t L = 0;
        while (L < 12 && ((2ull << L) - 1) * sizeof(K) <= 32768 && (2ull << L) <= a.n) ++L;
        const size_t smem = ((size_t)1 << L) * sizeof(K);
        auto kern = sorted_query_kernel<K>;
        int rc = persistent_grid(kern, smem, a.q, &grid);
        if (rc) return rc;
        kern<<<grid, kQueryThreads, smem, st>>>(A, a.n, L, Q, a.q, a.answers);
    } else if (a.layout == Q_BST) {
        // whole top levels: 2^T - 1 keys (a grouped batch over a large tree:
        // at most kBstGroupPinBytes of them, leaving room for more blocks)
        if (perm && tree_bytes >= (256ull << 20)) P = std::min<uint64_t>(P, kBstGroupPinBytes / sizeof(K));
        uint64_t top = 1;
        while (top * 2 + 1 <= P) top = top * 2 + 1;
        P = std::min<uint64_t>(top, a.n);
        size_t smem = P * sizeof(K);
        auto kern = bst_query_kernel<K>;
        int rc = persistent_grid(kern, smem, a.q, &grid);
        if (rc) return rc;
        kern<<<grid, kQueryThreads, smem, st>>>(A, a.n, P, Q, a.q, perm, a.answers);
    } else if (a.layout == Q_BTREE) {
        uint64_t top = 0, lvl = a.b;
        while (top + lvl <= P) {  // whole top levels: (b+1)^L - 1 keys
            top += lvl;
            if (lvl > UINT64_MAX / (a.b + 1)) break;
            lvl *= a.b + 1;
        }
        P = std::min<uint64_t>(top, a.n);
        size_t smem = P * sizeof(K);
        // a group of max(2, b * w / 64) lanes per query with 32-byte loads (b * w
        // = 64, 128 or 256 on a 32-byte aligned layout), else a thread per query
        // with 32-byte node loads (b * w a multiple of 32), else 16-byte ones
        // (b * w a multiple of 16), else a group of lanes per query with one key
        // per lane
        const uint64_t node_bytes = a.b * sizeof(K);
        const uintptr_t base = reinterpret_cast<uintptr_t>(A);
        int rc = TL_SUCCESS;
        bool done = false;
        auto v32 = [&](auto kern, bool pin) -> int {
            rc = persistent_grid(kern, pin ? smem : 0, a.q, &grid);
            if (rc) return rc;
            kern<<<grid, kQueryThreads, pin ? smem : 0, st>>>(A, a.n, pin ? P : 0, Q, a.q, a.answers);
            done = true;
            return TL_SUCCESS;
        };
        auto v16 = [&](auto kern) -> int {
            rc = persistent_grid(kern, 0, a.q, &grid);
            if (rc) return rc;
            kern<<<grid, kQueryThreads, 0, st>>>(A, a.n, a.b, Q, a.q, a.answers);
            done = true;
            return TL_SUCCESS;
        };
        const bool pin = g_query_variant == 5;
        auto grp = [&](auto kern, uint64_t lanes_per_query) -> int {
            rc = persistent_grid(kern, 0, a.q * lanes_per_query, &grid);
            if (rc) return rc;
            kern<<<grid, kQueryThreads, 0, st>>>(A, a.n, Q, a.q, a.answers);
            done = true;
            return TL_SUCCESS;
        };
        // default: nodes of 64, 128 or 256 bytes on a 32-byte aligned layout are
        // read by a group of max(2, node_bytes / 64) lanes.  Measured on B200,
        // 2^27 queries, q/s with 2 / 4 / 8 lanes per node against a thread per
        // query with 32-byte loads: b = 16 u64 over 5e8 keys 14.2e9 / 9.53e9 /
        // - against 6.54e9; b = 32 u64 over 2^28 keys 8.33e9 / 9.08e9 / 6.06e9
        // against 4.28e9; b = 16 u32 over 2^30 keys 17.7e9 against 11.7e9;
        // b = 8 u64 over 2^30 keys 12.7e9 against 8.56e9
        if ((base & 31) == 0 && g_query_variant != 2 && g_query_variant != 5 && g_query_variant != 6) {
            if (g_query_variant == 7) {  // one 32-byte load per lane
                switch (node_bytes) {
                    case 128: rc = grp(btree_query_group32_kernel<K, 128, 4>, 4); break;
                    case 256: rc = grp(btree_query_group32_kernel<K, 256, 8>, 8); break;
                    default: break;
                }
            }
            if (!done) {  // two 32-byte loads per lane (one for 64-byte nodes)
                switch (node_bytes) {
                    case 64: rc = grp(btree_query_group32_kernel<K, 64, 2>, 2); break;
                    case 128: rc = grp(btree_query_group32_kernel<K, 128, 2>, 2); break;
                    case 256: rc = grp(btree_query_group32_kernel<K, 256, 4>, 4); break;
                    default: break;
                }
            }
        }
        if (!done && (base & 31) == 0 && node_bytes % 32 == 0 && g_query_variant != 2) {
            switch (node_bytes) {
                case 32: rc = pin ? v32(btree_query_v32_kernel<K, 32, true>, true) : v32(btree_query_v32_kernel<K, 32, false>, false); break;
                case 64: rc = pin ? v32(btree_query_v32_kernel<K, 64, true>, true) : v32(btree_query_v32_kernel<K, 64, false>, false); break;
                case 128: rc = pin ? v32(btree_query_v32_kernel<K, 128, true>, true) : v32(btree_query_v32_kernel<K, 128, false>, false); break;
                case 256: rc = pin ? v32(btree_query_v32_kernel<K, 256, true>, true) : v32(btree_query_v32_kernel<K, 256, false>, false); break;
                default: break;
            }
        }
        if (!done && (base & 15) == 0 && node_bytes % 16 == 0) {
            switch (node_bytes / 16) {
                case 1: rc = v16(btree_query_vec_kernel<K, 1>); break;
                case 2: rc = v16(btree_query_vec_kernel<K, 2>); break;
                case 4: rc = v16(btree_query_vec_kernel<K, 4>); break;
                case 8: rc = v16(btree_query_vec_kernel<K, 8>); break;
                case 16: rc = v16(btree_query_vec_kernel<K, 16>); break;
                default: break;
            }
        }
        if (rc) return rc;
        if (done) {
            TL_CUDA_TRY(cudaGetLastError());
            return TL_SUCCESS;
        }
        int G = 1;
        while (G < 32 && (uint64_t)G < a.b) G <<= 1;
#define TL_BT(GG)                                                                          \
    case GG: {                                                                             \
        auto kern = btree_query_kernel<K, GG>;                                             \
        rc = persistent_grid(kern, smem, a.q * GG, &grid);                                 \
        if (rc) return rc;                                                                 \
        kern<<<grid, kQueryThreads, smem, st>>>(A, a.n, a.b, P, Q, a.q, a.answers);        \
        break;                                                                             \
    }
        switch (G) {
            TL_BT(1)
            TL_BT(2)
            TL_BT(4)
            TL_BT(8)
            TL_BT(16)
            TL_BT(32)
        }
#undef TL_BT
    } else {
        const uint32_t dmax = bit_length(a.n);
        if (dmax > 63) return TL_ERROR_UNSUPPORTED;
        const bool np = a.layout == Q_VEB_NP;
        const bool narrow = a.n < (1ull << 32);
        // QK columns of pos[] per thread; the layout's first positions pinned
        // in what is left of the block's shared-memory budget
        // one descent per thread: measured faster on B200 than two or four in
        // lock-step (2^27 queries over 2^30 - 1 u32 keys: 40.5 ms against 55.5
        // and 55.6; over 3e8 keys 36.6 against 49.0 and 49.3)
        const int qk = g_query_variant == 3 ? 2 : g_query_variant == 4 ? 4 : 1;
        const bool grouped = perm != nullptr && qk == 1;
        const int threads = grouped ? kVebGroupThreads : kVebThreads;
        const size_t budget = grouped ? kVebGroupBudget : qk == 1 ? 48 * 1024 : qk == 2 ? 72 * 1024 : 110 * 1024;
        const size_t pos_bytes = (size_t)dmax * qk * threads * (narrow ? 4 : 8);
        const size_t pin_budget = pos_bytes + kVebMinPin <= budget ? budget - pos_bytes : kVebMinPin;
        P = std::min<uint64_t>(a.n, pin_budget / sizeof(K));
        const size_t smem = (pos_bytes + 15) / 16 * 16 + P * sizeof(K);
        if (smem > 227 * 1024) return TL_ERROR_UNSUPPORTED;  // pos[] of a tree deeper than about 50 levels
        auto launch = [&](auto kern, int qpt) -> int {
            TL_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            int per_sm = 0;
            TL_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem));
            uint64_t g = (uint64_t)std::max(per_sm, 1) * query_sm_count();
            uint64_t need = (a.q + (uint64_t)qpt * threads - 1) / ((uint64_t)qpt * threads);
            unsigned gr = (unsigned)std::max<uint64_t>(1, std::min(g, need));
            kern<<<gr, threads, smem, st>>>(A, a.n, P, dmax, a.tables, np ? a.idx : nullptr,
                                                np ? a.table_idx : nullptr, np ? a.num_tables : 1u, Q, a.q, perm,
                                                a.answers);
            return TL_SUCCESS;
        };
        int rc;
        constexpr int T1 = kVebThreads, TG = kVebGroupThreads;
        if (grouped)
            rc = narrow ? launch(veb_query_kernel<K, uint32_t, 1, TG>, 1) : launch(veb_query_kernel<K, uint64_t, 1, TG>, 1);
        else if (qk == 1)
            rc = narrow ? launch(veb_query_kernel<K, uint32_t, 1, T1>, 1) : launch(veb_query_kernel<K, uint64_t, 1, T1>, 1);
        else if (qk == 2)
            rc = narrow ? launch(veb_query_kernel<K, uint32_t, 2, T1>, 2) : launch(veb_query_kernel<K, uint64_t, 2, T1>, 2);
        else
            rc = narrow ? launch(veb_query_kernel<K, uint32_t, 4, T1>, 4) : launch(veb_query_kernel<K, uint64_t, 4, T1>, 4);
        if (rc) return rc;
    }
    TL_CUDA_TRY(cudaGetLastError());
    return TL_SUCCESS;
}

int query(const QueryArgs &a, cudaStream_t st, float *ms) {
    if (a.q == 0) {
        if (ms) *ms = 0.f;
        return TL_SUCCESS;
    }
    if (!a.queries || !a.answers) return TL_ERROR_INVALID_VALUE;
    if (a.n == 0) {
        TL_CUDA_TRY(cudaMemsetAsync(a.answers, 0, a.q * sizeof(uint64_t), st));
        if (ms) *ms = 0.f;
        return sync_and_check(st);
    }
    if (!a.layout_keys) return TL_ERROR_INVALID_VALUE;
    if (a.layout == Q_BTREE && a.b == 0) return TL_ERROR_INVALID_VALUE;
    if ((a.layout == Q_VEB || a.layout == Q_VEB_NP) && !a.tables) return TL_ERROR_INVALID_VALUE;
    if (a.layout == Q_VEB_NP && (!a.idx || !a.table_idx || a.num_tables == 0)) return TL_ERROR_INVALID_VALUE;
    EventTimer timer(ms != nullptr, st);
    timer.start();
    int rc = a.key_bytes == 8 ? launch_query<uint64_t>(a, st) : launch_query<uint32_t>(a, st);
    timer.stop();
    if (rc) return rc;
    if (ms) {
        rc = sync_and_check(st);
        if (rc) return rc;
        *ms = timer.elapsed();
    }
    return TL_SUCCESS;
}

}  // namespace tl
