// The reference's cycle-leader algorithm family as a selectable variant of the
// permutation (TL_ALGO_CYCLES: B-tree any b, BST as the B-tree with b = 1,
// mvEB; TL_ALGO_HYBRID: the BST's last level by cycles, its perfect part by
// involutions), for ablations and as a third route to the same layouts.
//
// The family (Berney, Casanova, Karsin, Sitchinava, "Beyond binary search:
// parallel in-place construction of implicit search tree layouts", IPDPS 2018)
// builds every layout from one primitive, the equidistant gather: in an array
// of r groups of (l leaf chunks, 1 root chunk) of c keys each (r <= l),
// followed by trailing leaf chunks, bring the r root chunks to the front in
// order and keep the leaf chunks in order behind them.  It takes two steps:
//  1. r cycle-leader walks: walk i moves the chunks at i, i + l, ..., i + i l
//     one place along (chunk i + (i + 1) l, root i, ends at chunk i);
//  2. r rotations: leaf group i (chunks r + i l .. r + (i + 1) l) rotated
//     right by r - i chunks, by two reversal passes.
// The layouts follow the reference's recursions, restated as host code that
// emits these steps (equidistant gathers of partitions, chunks, rotations):
//  - B-tree (gpu/src/btree-cycles.cuh:31-104, cpu/src/btree-cycles.h:26-96):
//    a non-perfect tree first gathers its last level (the extended gather for
//    n = m (b + 1), gpu/src/cycles.cuh:707-960) and rotates the
//    remaining internal keys behind the gathered separators; then, per level,
//    the extended gather for n = (b + 1)^d - 1 (gpu/src/cycles.cuh:997-1100:
//    rounds of chunk size c = 1, b + 1, (b + 1)^2 ... over partitions of
//    (b + 1)^2 c keys) and the next level on the n / (b + 1) gathered keys;
//  - mvEB (gpu/src/mveb-cycles.cuh:31-441): gather the root keys (one per
//    full bottom tree), rotate the missing roots into place for a non-perfect
//    tree, lay out the bottom trees as balanced vEB trees (rounds of gathers
//    over equal partitions down to the 255 / 15 / 3-key base cases), recurse
//    on the root tree and on the incomplete last bottom tree;
//  - hybrid BST (gpu/src/bst-hybrid.cuh:93-148): the last level as the B-tree
//    with b = 1, the perfect rest by the involutions (variants.cu).
// Sibling subproblems of the same shape become one batched step (instances at
// base + sum_d digit_d * stride_d), so each step is one set of launches
// whatever the number of partitions; steps run in the recursion's order.  The
// same step list runs on the host (tl_debug_emulate_algorithm) for the CPU tests.
#include <algorithm>
#include <vector>

#include "internal.h"
#include "tl_common.cuh"

namespace tl {

constexpr int kCycThreads = 256;
constexpr int kCycDims = 8;

enum CycKind : uint32_t { CYC_GATHER = 0, CYC_ROTATE = 1 };

// One step over `inst` instances, instance j at base + sum_d digit_d(j) str[d]
// (digits of j in the mixed radix cnt[], the last dimension fastest).
//  gather: r roots, l leaves, chunks of c keys (the equidistant gather above);
//  rotate: a = length, k = right shift.
struct CycOp {
    uint32_t kind = CYC_GATHER, nd = 0;
    uint64_t base = 0, r = 0, l = 0, c = 1;
    uint64_t cnt[kCycDims] = {}, str[kCycDims] = {};
    uint64_t inst = 1;
};

TL_HD uint64_t cyc_offset(const CycOp &op, uint64_t j) {
    uint64_t off = op.base;
    for (int d = (int)op.nd - 1; d >= 0; --d) {
        const uint64_t q = j / op.cnt[d];
        off += (j - q * op.cnt[d]) * op.str[d];
        j = q;
    }
    return off;
}

// ---------------------------------------------------------------- step lists
// Replication context of a recursion: the instances a subproblem stands for.
struct Reps {
    int nd = 0;
    uint64_t cnt[kCycDims] = {}, str[kCycDims] = {};
    bool overflow = false;
    // `k` copies at stride s inside every current instance; contiguous nests
    // (an outer stride equal to the inner span) fold into one dimension
    Reps push(uint64_t k, uint64_t s) const {
        Reps o = *this;
        if (k <= 1) return o;
        if (o.nd > 0 && o.str[o.nd - 1] == k * s) {
            o.cnt[o.nd - 1] *= k;
            o.str[o.nd - 1] = s;
            return o;
        }
        if (o.nd == kCycDims) {
            o.overflow = true;
            return o;
        }
        o.cnt[o.nd] = k;
        o.str[o.nd] = s;
        ++o.nd;
        return o;
    }
};

struct CycList {
    std::vector<CycOp> ops;
    bool overflow = false;
    void gather(const Reps &R, uint64_t base, uint64_t r, uint64_t l, uint64_t c) {
        if (r == 0 || l == 0 || c == 0) return;
        add(R, CYC_GATHER, base, r, l, c);
    }
    void rotate(const Reps &R, uint64_t base, uint64_t a, uint64_t k) {
        if (a < 2 || k % a == 0) return;
        add(R, CYC_ROTATE, base, a, k % a, 1);
    }
    void add(const Reps &R, uint32_t kind, uint64_t base, uint64_t r, uint64_t l, uint64_t c) {
        if (R.overflow) {
            overflow = true;
            return;
        }
        CycOp op;
        op.kind = kind;
        op.base = base;
        op.r = r;
        op.l = l;
        op.c = c;
        op.nd = (uint32_t)R.nd;
        op.inst = 1;
        for (int d = 0; d < R.nd; ++d) {
            op.cnt[d] = R.cnt[d];
            op.str[d] = R.str[d];
            op.inst *= R.cnt[d];
        }
        ops.push_back(op);
    }
};

// Extended equidistant gather for n = m (b + 1) (gpu/src/cycles.cuh:707-960):
// every (b + 1)-th key to the front, the rest in order behind.  Bottom-up
// rounds of chunk size c = 1, k, k^2, ... (k = b + 1): in every full partition
// of k^2 c keys the b root chunks gathered, in the last, incomplete partition
// the r_c - 1 root chunks it holds, and the roots gathered so far (r keys)
// rotated forward past that partition's leaves.
static void emit_gather2(CycList &L, uint64_t n, uint64_t b) {
    const uint64_t k = b + 1;
    uint64_t c = 1, m = k * k, P = (n + 1) / m;
    uint64_t r = ((n + 1) % m) / k + 1;  // root keys of the last, incomplete partition, plus one
    const Reps R;
    if (P == 0) {
        L.gather(R, 0, r - 1, b, 1);
        return;
    }
    L.gather(R.push(P, m), 0, b, b, 1);
    if (r > 1) L.gather(R, m * P, r - 1, b, 1);
    auto next = [&](uint64_t &rc) {
        rc = P % k;
        if (P < k) --rc;
        P /= k;
        m *= k;
        c *= k;
    };
    uint64_t rc;
    next(rc);
    while (P >= 1) {
        L.gather(R.push(P, m), c - 1, b, b, c);
        if (rc > 1) L.gather(R, P * m - 1 + c, rc - 1, b, c);
        if (rc > 0) L.rotate(R, P * m - 1 + rc * c, rc * b * c + r, r);
        r += rc * c;
        next(rc);
    }
    if (rc > 0) L.gather(R, c - 1, rc, b, c);
    L.rotate(R, c - 1 + rc * c, (rc + 1) * b * c + r, r);
}

// Extended equidistant gather for n = (b + 1)^d - 1 (gpu/src/cycles.cuh:997-1100):
// rounds of chunk size c over partitions of (b + 1)^2 c keys.
static void emit_gather_perfect(CycList &L, uint64_t n, uint64_t b) {
    const uint64_t k = b + 1;
    Reps R;
    for (uint64_t c = 1;; c *= k) {
        const uint64_t m = k * k * c;
        if (m > n + 1) break;
        L.gather(R.push((n + 1) / m, m), c - 1, b, b, c);
        if (c > (n + 1) / (k * k * k)) break;
    }
}

static void emit_btree(CycList &L, uint64_t n, uint64_t b) {
    const uint64_t k = b + 1;
    uint32_t h = 0;
    uint64_t p = 1;
    while (p <= n / k) {
        p *= k;
        ++h;
    }
    uint64_t top = n;
    uint32_t d = h + 1;
    if (n != p * k - 1) {  // non-perfect: the last level first (btree-cycles.cuh:31-60)
        const uint64_t ni = p - 1, nl = n - ni;
        const uint64_t r = nl % b, l = nl - r, i = l / b;
        emit_gather2(L, l + i, b);
        L.rotate(Reps(), i, nl + ni - i, ni - i);
        top = ni;
        d = h;
    }
    for (; d > 1; --d) {  // btree-cycles.cuh:63-70
        emit_gather_perfect(L, top, b);
        top /= k;
    }
}

// BST leaves for the hybrid (gpu/src/bst-hybrid.cuh:71-91); returns the size of
// the perfect front part, laid out by the involutions afterwards.
static uint64_t emit_bst_leaves(CycList &L, uint64_t n) {
    uint32_t h = 0;
    while (h + 1 < 64 && (1ull << (h + 1)) <= n) ++h;
    if (n == (1ull << (h + 1)) - 1) return n;
    const uint64_t ni = (1ull << h) - 1, nl = n - ni;
    emit_gather2(L, 2 * nl, 1);
    L.rotate(Reps(), nl, ni, ni - nl);
    return ni;
}

static bool is_pow2(uint64_t x) { return x && !(x & (x - 1)); }

static uint64_t isqrt(uint64_t m) {
    uint64_t s = 0;
    for (int bit = 31; bit >= 0; --bit) {
        const uint64_t t = s | (1ull << bit);
        if (t * t <= m) s = t;
    }
    return s;
}

// Balanced vEB trees of m = 2^d - 1 keys (d a power of two), all n / m of them
// (gpu/src/mveb-cycles.cuh:31-226): rounds of root gathers down to the 255 /
// 15 / 3-key base cases, each itself a chain of gathers.
static void emit_balanced(CycList &L, const Reps &R, uint64_t base, uint64_t n, uint64_t m, uint32_t d) {
    if (d <= 1 || m <= 1 || n < m) return;
    while (d > 8) {
        const uint64_t k = isqrt(m);
        L.gather(R.push(n / m, m), base, k, k, 1);
        m = k;
        d /= 2;
    }
    if (d == 8) {
        L.gather(R.push(n / 255, 255), base, 15, 15, 1);
        d = 4;
    }
    if (d == 4) {
        L.gather(R.push(n / 15, 15), base, 3, 3, 1);
        d = 2;
    }
    if (d == 2) L.gather(R.push(n / 3, 3), base, 1, 1, 1);
}

static void veb_split(uint32_t d, uint32_t &root_d, uint32_t &leaf_d) {
    root_d = (d - 2) / 2 + 1;
    leaf_d = d - root_d;
    if (!is_pow2(leaf_d)) {  // the modified split: bottoms of a power-of-two height
        uint32_t p = 1;
        while (p < leaf_d) p <<= 1;
        leaf_d = p;
        root_d = d - leaf_d;
    }
}

static void emit_mveb_perfect(CycList &L, const Reps &R, uint64_t base, uint64_t n, uint32_t d);

static void emit_mveb_root(CycList &L, const Reps &R, uint64_t base, uint64_t r, uint32_t root_d) {
    if (is_pow2(root_d))
        emit_balanced(L, R, base, r, r, root_d);
    else
        emit_mveb_perfect(L, R, base, r, root_d);
}

// permutevEB (gpu/src/mveb-cycles.cuh:231-290): n = 2^d - 1, d not a power of two.
static void emit_mveb_perfect(CycList &L, const Reps &R, uint64_t base, uint64_t n, uint32_t d) {
    if (n <= 1) return;
    uint32_t root_d, leaf_d;
    veb_split(d, root_d, leaf_d);
    const uint64_t r = (1ull << root_d) - 1, l = (1ull << leaf_d) - 1;
    L.gather(R, base, r, l, 1);
    emit_balanced(L, R, base + r, n - r, l, leaf_d);
    emit_mveb_root(L, R, base, r, root_d);
}

// permutevEB_nonperfect (gpu/src/mveb-cycles.cuh:294-414): 2^(d-1) - 1 < n < 2^d - 1.
static void emit_mveb_nonperfect(CycList &L, const Reps &R, uint64_t base, uint64_t n, uint32_t d) {
    if (n <= 1) return;
    uint32_t root_d, leaf_d;
    veb_split(d, root_d, leaf_d);
    const uint64_t r = (1ull << root_d) - 1, l = (1ull << leaf_d) - 1;
    const uint64_t num_full = (n - r) / l, inc_n = n - r - num_full * l;
    L.gather(R, base, num_full, l, 1);
    if (num_full < r) L.rotate(R, base + num_full, n - num_full, r - num_full);
    if (root_d == leaf_d) {
        emit_balanced(L, R, base, n - inc_n, r, root_d);
    } else {
        emit_balanced(L, R, base + r, num_full * l, l, leaf_d);
        emit_mveb_root(L, R, base, r, root_d);
    }
    if (inc_n > 0) {
        uint32_t inc_d = 0;
        while ((1ull << inc_d) <= inc_n) ++inc_d;  // floor(log2 inc_n) + 1
        if (inc_n != (1ull << inc_d) - 1)
            emit_mveb_nonperfect(L, R, base + n - inc_n, inc_n, inc_d);
        else
            emit_mveb_root(L, R, base + n - inc_n, inc_n, inc_d);
    }
}

static void emit_mveb(CycList &L, uint64_t n) {
    uint32_t d = 0;
    while ((1ull << d) <= n) ++d;  // floor(log2 n) + 1
    if (n != (1ull << d) - 1)
        emit_mveb_nonperfect(L, Reps(), 0, n, d);
    else
        emit_mveb_root(L, Reps(), 0, n, d);
}

// ---------------------------------------------------------------- host replay
// Same steps and the same per-step semantics as the kernels: the walks of a
// gather, then its rotations; instances and walks are independent.
static void host_rotate(uint64_t *A, uint64_t a, uint64_t k) {
    std::reverse(A, A + a);
    std::reverse(A, A + k);
    std::reverse(A + k, A + a);
}

static void host_run(const CycList &L, uint64_t *A) {
    for (const CycOp &op : L.ops) {
        for (uint64_t j = 0; j < op.inst; ++j) {
            uint64_t *a = A + cyc_offset(op, j);
            if (op.kind == CYC_ROTATE) {
                host_rotate(a, op.r, op.l);
                continue;
            }
            const uint64_t r = op.r, l = op.l, c = op.c;
            for (uint64_t i = 0; i < r; ++i)
                for (uint64_t t = 0; t < c; ++t) {
                    uint64_t q = (i + (i + 1) * l) * c + t;
                    const uint64_t tmp = a[q];
                    for (; q > i * c + t; q -= l * c) a[q] = a[q - l * c];
                    a[i * c + t] = tmp;
                }
            for (uint64_t i = 0; i < r; ++i) host_rotate(a + (r + i * l) * c, l * c, (r - i) * c);
        }
    }
}

// ---------------------------------------------------------------- kernels
// Walks: one per (instance, root i, key t of the chunk).
template <typename K>
__global__ void __launch_bounds__(kCycThreads) cyc_walk_kernel(K *A, const __grid_constant__ CycOp op) {
    const uint64_t per = op.r * op.c, work = op.inst * per;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t w = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; w < work; w += stride) {
        const uint64_t j = w / per, rem = w - j * per, i = rem / op.c, t = rem - i * op.c;
        K *a = A + cyc_offset(op, j);
        const uint64_t lc = op.l * op.c, lo = i * op.c + t;
        uint64_t q = (i + (i + 1) * op.l) * op.c + t;
        const K tmp = a[q];
        for (; q > lo; q -= lc) a[q] = a[q - lc];
        a[lo] = tmp;
    }
}

// Segment s of instance j for the rotation passes: gathers rotate their r leaf
// groups (l c keys, right by (r - i) c), rotations their one array.
__device__ __forceinline__ void cyc_segment(const CycOp &op, uint64_t s, uint64_t &start, uint64_t &len,
                                            uint64_t &k) {
    if (op.kind == CYC_ROTATE) {
        start = 0;
        len = op.r;
        k = op.l;
    } else {
        start = (op.r + s * op.l) * op.c;
        len = op.l * op.c;
        k = ((op.r - s) * op.c) % len;
    }
}

// pass 0: each segment reversed whole; pass 1: its first k and last len - k
// keys reversed (a right rotation by k).  One thread per swapped pair.
template <typename K>
__global__ void __launch_bounds__(kCycThreads) cyc_reverse_kernel(K *A, const __grid_constant__ CycOp op, int pass) {
    const uint64_t segs = op.kind == CYC_ROTATE ? 1 : op.r;
    const uint64_t maxlen = op.kind == CYC_ROTATE ? op.r : op.l * op.c;
    const uint64_t per = maxlen / 2, work = op.inst * segs * per;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t w = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; w < work; w += stride) {
        const uint64_t js = w / per, x = w - js * per, j = js / segs, s = js - j * segs;
        uint64_t start, len, k;
        cyc_segment(op, s, start, len, k);
        if (k == 0) continue;
        K *a = A + cyc_offset(op, j) + start;
        uint64_t p, q;
        if (pass == 0) {
            p = x;
            q = len - 1 - x;
        } else if (x < k / 2) {
            p = x;
            q = k - 1 - x;
        } else if (x - k / 2 < (len - k) / 2) {
            const uint64_t y = x - k / 2;
            p = k + y;
            q = len - 1 - y;
        } else {
            continue;
        }
        const K tmp = a[p];
        a[p] = a[q];
        a[q] = tmp;
    }
}

static unsigned cyc_grid(uint64_t work) {
    return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((work + kCycThreads - 1) / kCycThreads, 148ull * 16));
}

template <typename K>
static int run_ops(const CycList &L, K *A, cudaStream_t st) {
    for (const CycOp &op : L.ops) {
        if (op.kind == CYC_GATHER) {
            cyc_walk_kernel<K><<<cyc_grid(op.inst * op.r * op.c), kCycThreads, 0, st>>>(A, op);
            TL_CUDA_TRY(cudaGetLastError());
        }
        const uint64_t pairs = op.inst * (op.kind == CYC_ROTATE ? op.r / 2 : op.r * (op.l * op.c / 2));
        if (pairs == 0) continue;
        for (int pass = 0; pass < 2; ++pass) {
            cyc_reverse_kernel<K><<<cyc_grid(pairs), kCycThreads, 0, st>>>(A, op, pass);
            TL_CUDA_TRY(cudaGetLastError());
        }
    }
    return TL_SUCCESS;
}

// ---------------------------------------------------------------- entry points
// The step list of a layout by the cycle-leader family; for the hybrid BST the
// steps of its last level and, in *perfect, the size of the front part the
// involutions finish.
static int cycles_list(int layout, int algorithm, uint64_t n, uint64_t b, CycList &L, uint64_t *perfect) {
    if (perfect) *perfect = 0;
    if (algorithm == TL_ALGO_HYBRID) {
        if (layout != TL_LAYOUT_BST) return TL_ERROR_UNSUPPORTED;
        const uint64_t ni = emit_bst_leaves(L, n);
        if (perfect) *perfect = ni;
    } else if (layout == TL_LAYOUT_BST) {
        emit_btree(L, n, 1);
    } else if (layout == TL_LAYOUT_BTREE) {
        emit_btree(L, n, b);
    } else if (layout == TL_LAYOUT_MVEB) {
        emit_mveb(L, n);
    } else {
        return TL_ERROR_UNSUPPORTED;  // the standard vEB: the reference has it on the CPU only
    }
    return L.overflow ? TL_ERROR_UNSUPPORTED : TL_SUCCESS;
}

int permute_cycles(int layout, int algorithm, void *dev_A, uint64_t n, uint64_t b, uint32_t key_bytes,
                   cudaStream_t st, uint64_t *perfect) {
    CycList L;
    const int rc = cycles_list(layout, algorithm, n, b, L, perfect);
    if (rc) return rc;
    return key_bytes == 8 ? run_ops(L, static_cast<uint64_t *>(dev_A), st)
                          : run_ops(L, static_cast<uint32_t *>(dev_A), st);
}

int emulate_cycles(int layout, int algorithm, uint64_t n, uint64_t b, uint64_t *A, uint64_t *perfect,
                   uint64_t *steps) {
    CycList L;
    const int rc = cycles_list(layout, algorithm, n, b, L, perfect);
    if (rc) return rc;
    host_run(L, A);
    if (steps) *steps = L.ops.size();
    return TL_SUCCESS;
}

}  // namespace tl
