// Learned-start exact B-tree query (no counterpart in the reference).
//
// A two-stage rank model predicts the sorted rank of a key: an FP32 root MLP
// 1 -> 32 -> 32 -> 1 over the normalised key picks one of L linear leaf segments;
// the leaf maps the key to a rank and carries eps, the largest rank error over
// the keys it was fitted on.  The query starts its B-tree descent at the deepest
// subtree whose in-order rank range covers [rank - eps, rank + eps].  Answers
// stay exact: a hit is a hit; a miss is only accepted when the subtree held keys
// on both sides of the query (so the key, if present, would be in it); every
// other case falls back to the plain search from the root.
//
// Everything here is hand-written CUDA: the training batch sampler, the forward
// and backward passes (per-block partial gradients reduced in a fixed order, so
// training is deterministic), Adam, the leaf fit, the eps pass, inference and
// the query.
#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstring>
#include <memory>
#include <mutex>
#include <vector>

#include "geometry.cuh"
#include "internal.h"
#include "learned.h"

namespace tl {

constexpr int H = TL_RMI_HIDDEN;
constexpr int kParams = H + H + H * H + H + H + 1;  // w1 b1 w2 b2 w3 b3
constexpr int kTrainThreads = 64;                  // samples per training block

// The trained root network evaluated through its exact piecewise-linear form.
// With one input and ReLU hidden layers the network is a continuous
// piecewise-linear function of x: the first layer's units switch at most once
// each (at x = -b1 / w1), and between two such points every second-layer
// unit is affine in x and switches at most once more.  compile_root lists the
// pieces (at most 33 * 33; start of each piece, slope, intercept) on the host
// in double precision; inference finds x's piece by binary search in shared
// memory and takes one FMA, where the layer-by-layer form takes about 1 100.
// Every inference step - the leaf fit, the eps pass, prediction and the
// queries - uses this one evaluator, so each leaf's eps bounds exactly what
// the queries see.  Training itself runs the network layer by layer
// (rmi_grad_kernel).
constexpr uint32_t kMaxPieces = 1152;  // >= 33 * 33
constexpr uint32_t kGridCells = 1024;  // uniform index over [0, 1]

struct RootPieces {
    uint32_t count;
    float x0[kMaxPieces];  // piece k covers [x0[k], x0[k + 1]); x0[0] = 0
    float s[kMaxPieces], t[kMaxPieces];
    // first[c]: the piece holding c / kGridCells, so an x in cell c lies in a
    // piece of first[c] .. first[c + 1]
    uint16_t first[kGridCells + 1];
};

struct ModelParams {  // kernel-parameter copy of the inference model (constant bank)
    RootPieces root;
    float x_lo, x_scale;
    uint32_t log_feature, num_leaves;
};

static void compile_root(const tl_rank_model &m, RootPieces &rp) {
    std::vector<double> bp = {0.0, 1.0};
    for (int i = 0; i < H; ++i)
        if (m.w1[i] != 0.f) {
            const double x = -(double)m.b1[i] / (double)m.w1[i];
            if (x > 0.0 && x < 1.0) bp.push_back(x);
        }
    std::sort(bp.begin(), bp.end());
    bp.erase(std::unique(bp.begin(), bp.end()), bp.end());
    rp.count = 0;
    std::vector<double> sub;
    double A[H], C[H];
    for (size_t iv = 0; iv + 1 < bp.size(); ++iv) {
        const double a = bp[iv], c = bp[iv + 1], mid = 0.5 * (a + c);
        for (int j = 0; j < H; ++j) {  // second-layer pre-activation = A_j x + C_j on (a, c)
            A[j] = 0.0;
            C[j] = (double)m.b2[j];
            for (int i = 0; i < H; ++i)
                if ((double)m.w1[i] * mid + (double)m.b1[i] > 0.0) {
                    A[j] += (double)m.w2[j][i] * (double)m.w1[i];
                    C[j] += (double)m.w2[j][i] * (double)m.b1[i];
                }
        }
        sub.assign({a, c});
        for (int j = 0; j < H; ++j)
            if (A[j] != 0.0) {
                const double x = -C[j] / A[j];
                if (x > a && x < c) sub.push_back(x);
            }
        std::sort(sub.begin(), sub.end());
        sub.erase(std::unique(sub.begin(), sub.end()), sub.end());
        for (size_t k = 0; k + 1 < sub.size(); ++k) {
            const double m2 = 0.5 * (sub[k] + sub[k + 1]);
            double S = 0.0, T = (double)m.b3;
            for (int j = 0; j < H; ++j)
                if (A[j] * m2 + C[j] > 0.0) {
                    S += (double)m.w3[j] * A[j];
                    T += (double)m.w3[j] * C[j];
                }
            if (rp.count == kMaxPieces) return;  // cannot happen: at most 33 * 33 pieces
            rp.x0[rp.count] = (float)sub[k];
            rp.s[rp.count] = (float)S;
            rp.t[rp.count] = (float)T;
            ++rp.count;
        }
    }
    rp.x0[0] = 0.f;
    uint32_t k = 0;
    for (uint32_t c = 0; c <= kGridCells; ++c) {
        const float e = (float)c / (float)kGridCells;  // exact: kGridCells is a power of two
        while (k + 1 < rp.count && rp.x0[k + 1] <= e) ++k;
        rp.first[c] = (uint16_t)k;
    }
}

static void model_to_flat(const tl_rank_model &m, float *w);

// Compiled roots of the last few models seen, keyed by their root weights:
// compiling (host, double precision, up to 33 x 33 pieces) costs more than a
// small query batch, and one model serves many batches.
struct RootCacheEntry {
    float w[kParams];  // the weights the pieces were compiled from
    RootPieces rp;
    uint64_t stamp;
};
constexpr size_t kRootCacheEntries = 4;
static std::mutex g_root_mu;
static std::vector<std::unique_ptr<RootCacheEntry>> g_root_cache;
static uint64_t g_root_clock = 0;

static void compiled_root(const tl_rank_model &m, RootPieces &out) {
    float w[kParams];
    model_to_flat(m, w);
    std::lock_guard<std::mutex> lock(g_root_mu);
    RootCacheEntry *hit = nullptr;
    for (auto &e : g_root_cache)
        if (!std::memcmp(e->w, w, sizeof w)) hit = e.get();
    if (!hit) {
        std::unique_ptr<RootCacheEntry> e(new RootCacheEntry);
        std::memcpy(e->w, w, sizeof w);
        compile_root(m, e->rp);
        if (g_root_cache.size() >= kRootCacheEntries) {
            size_t old = 0;
            for (size_t k = 1; k < g_root_cache.size(); ++k)
                if (g_root_cache[k]->stamp < g_root_cache[old]->stamp) old = k;
            g_root_cache.erase(g_root_cache.begin() + (long)old);
        }
        hit = e.get();
        g_root_cache.push_back(std::move(e));
    }
    hit->stamp = ++g_root_clock;
    out = hit->rp;
}

static ModelParams to_params(const tl_rank_model &m) {
    ModelParams p;
    compiled_root(m, p.root);
    p.x_lo = (float)m.x_lo;
    p.x_scale = (float)m.x_scale;
    p.log_feature = m.log_feature;
    p.num_leaves = m.num_leaves;
    return p;
}

// The pieces in shared memory (every thread of the block, before any use).
struct PiecesSmem {
    float x0[kMaxPieces], s[kMaxPieces], t[kMaxPieces];
    uint16_t first[kGridCells + 1];
};

__device__ __forceinline__ void stage_pieces(const ModelParams &p, PiecesSmem &sp) {
    for (uint32_t k = threadIdx.x; k < p.root.count; k += blockDim.x) {
        sp.x0[k] = p.root.x0[k];
        sp.s[k] = p.root.s[k];
        sp.t[k] = p.root.t[k];
    }
    for (uint32_t c = threadIdx.x; c <= kGridCells; c += blockDim.x) sp.first[c] = p.root.first[c];
    __syncthreads();
}

// The root's output at x in [0, 1]: the last piece starting at or below x,
// found from x's grid cell (usually no further step; a binary search where
// several pieces start inside one cell).
TL_HD float pieces_eval(const float *x0, const float *s, const float *t, const uint16_t *first, float x) {
    const uint32_t cf = (uint32_t)(x * (float)kGridCells);
    const uint32_t c = cf < kGridCells ? cf : kGridCells - 1;
    uint32_t lo = first[c], hi = first[c + 1];
    while (lo < hi) {
        const uint32_t mid = (lo + hi + 1) >> 1;
        if (x0[mid] <= x)
            lo = mid;
        else
            hi = mid - 1;
    }
    return fmaf(s[lo], x, t[lo]);
}

// Normalised feature of a key, in [0, 1] over the trained key range:
// f = log2(key + 1) (FP32) or the key itself, x = (f - x_lo) * x_scale clamped.
// Training, the segment fit and the queries all evaluate it with this one
// function (feature_of is the same arithmetic for training's parameter struct).
__device__ __forceinline__ float feature_x(uint32_t log_feature, float x_lo, float x_scale, uint64_t key) {
    const float f = log_feature ? log2f((float)key + 1.0f) : (float)key;
    const float x = (f - x_lo) * x_scale;
    return x < 0.f ? 0.f : (x > 1.f ? 1.f : x);
}

__device__ __forceinline__ float feature(const ModelParams &p, uint64_t key) {
    return feature_x(p.log_feature, p.x_lo, p.x_scale, key);
}

__device__ __forceinline__ uint32_t leaf_of(const ModelParams &p, float out) {
    float f = out * (float)p.num_leaves;
    if (!(f > 0.f)) return 0;  // also catches NaN
    uint32_t l = (uint32_t)f;
    return l < p.num_leaves ? l : p.num_leaves - 1;
}

// The root's output (use_net) or, for the leaf-only ablation, x itself.
__device__ __forceinline__ float root_eval(const ModelParams &p, const PiecesSmem &sp, float x, bool use_net) {
    return use_net ? pieces_eval(sp.x0, sp.s, sp.t, sp.first, x) : x;
}

static_assert(sizeof(tl_rank_leaf) == 32 && offsetof(tl_rank_leaf, slope) == 16 &&
                  offsetof(tl_rank_leaf, eps_lo) == 20 && offsetof(tl_rank_leaf, empty) == 28,
              "load_leaf reads the segment entry as four 64-bit words");

// A segment entry from its four 64-bit words (its layout in memory).
__device__ __forceinline__ tl_rank_leaf leaf_from_words(const uint64_t (&w)[4]) {
    tl_rank_leaf lf;
    lf.kmin = w[0];
    lf.base = w[1];
    lf.slope = __uint_as_float((uint32_t)w[2]);
    lf.eps_lo = (uint32_t)(w[2] >> 32);
    lf.eps_hi = (uint32_t)w[3];
    lf.empty = (uint32_t)(w[3] >> 32);
    return lf;
}

// A segment entry (32 bytes) in one load where the table is 32-byte aligned.
__device__ __forceinline__ tl_rank_leaf load_leaf(const tl_rank_leaf *__restrict__ leaves, uint32_t l,
                                                  bool aligned32) {
    if (!aligned32) return leaves[l];
    uint64_t w[4];
    ldg32(reinterpret_cast<const uint64_t *>(leaves + l), w);
    return leaf_from_words(w);
}

// Rank prediction of a segment, clamped to [0, n).
// The segment's base rank stays an integer and only the offset within the
// segment is FP32 (the base itself in FP32 would round to 64 ranks near 2^30,
// and that rounding would widen every window).
__device__ __forceinline__ uint64_t leaf_predict(const tl_rank_leaf &lf, uint64_t key, uint64_t n) {
    const float off = key > lf.kmin ? (float)(key - lf.kmin) : 0.f;
    const float d = lf.slope * off;  // >= 0: slopes are non-negative
    const uint64_t ri = lf.base + (d > 0.f ? (uint64_t)(d + 0.5f) : 0ull);
    return ri < n ? ri : n - 1;
}

// splitmix64 (Steele, Lea, Flood, OOPSLA 2014) for the training sampler.
TL_HD uint64_t mix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

// ---------------------------------------------------------------- training
// Flat parameter order: w1[H] b1[H] w2[H][H] b2[H] w3[H] b3.
// Per block: forward + backward of kTrainThreads samples with the current
// weights (read from `w`, staged in shared memory), gradient of the mean
// squared error over the batch summed over the block's samples in a fixed
// order, written to partial[block][kParams].  Samples come either from (x, y)
// arrays or from the sorted keys (rank drawn by a hash of (seed, index)).
struct Feature {
    float x_lo, x_scale;
    uint32_t log_feature;
};

__device__ __forceinline__ float feature_of(const Feature &f, uint64_t key) {
    return feature_x(f.log_feature, f.x_lo, f.x_scale, key);
}

__global__ void __launch_bounds__(kTrainThreads)
rmi_grad_kernel(const float *__restrict__ w, Feature fe, const float *__restrict__ xs,
                const float *__restrict__ ys, const uint64_t *__restrict__ keys, uint64_t n, uint64_t seed,
                uint32_t m, float inv_m, float *__restrict__ partial, float *__restrict__ loss_partial) {
    __shared__ float sw[kParams];
    __shared__ float s_h1[kTrainThreads][H + 1];
    __shared__ float s_h2[kTrainThreads][H + 1];
    __shared__ float s_dz1[kTrainThreads][H + 1];
    __shared__ float s_dz2[kTrainThreads][H + 1];
    __shared__ float s_x[kTrainThreads];
    __shared__ float s_dout[kTrainThreads];
    __shared__ float s_loss[kTrainThreads];
    const uint32_t t = threadIdx.x;
    for (int k = t; k < kParams; k += kTrainThreads) sw[k] = w[k];
    __syncthreads();
    const float *w1 = sw, *b1 = sw + H, *w2 = sw + 2 * H, *b2 = sw + 2 * H + H * H, *w3 = b2 + H;
    const float b3 = w3[H];
    const uint64_t gi = (uint64_t)blockIdx.x * kTrainThreads + t;
    const bool valid = gi < m;
    float x = 0.f, y = 0.f;
    if (valid) {
        if (xs) {
            x = xs[gi];
            y = ys[gi];
        } else {
            const uint64_t r = mix64(seed ^ mix64(gi)) % n;
            x = feature_of(fe, keys[r]);
            y = ((float)r + 0.5f) / (float)n;
        }
    }
    // forward; ReLU masks kept as bits, activations in shared memory
    float h1[H];
    uint32_t mask1 = 0, mask2 = 0;
#pragma unroll
    for (int i = 0; i < H; ++i) {
        const float z = fmaf(w1[i], x, b1[i]);
        h1[i] = fmaxf(z, 0.f);
        mask1 |= (z > 0.f ? 1u : 0u) << i;
        s_h1[t][i] = h1[i];
    }
    float out = b3;
    for (int j = 0; j < H; ++j) {
        float a = b2[j];
#pragma unroll
        for (int i = 0; i < H; ++i) a = fmaf(w2[j * H + i], h1[i], a);
        mask2 |= (a > 0.f ? 1u : 0u) << j;
        const float h2 = fmaxf(a, 0.f);
        s_h2[t][j] = h2;
        out = fmaf(w3[j], h2, out);
    }
    // backward
    const float diff = out - y;
    const float dout = valid ? 2.f * diff * inv_m : 0.f;
    s_loss[t] = valid ? diff * diff * inv_m : 0.f;
    s_x[t] = x;
    s_dout[t] = dout;
#pragma unroll
    for (int j = 0; j < H; ++j) s_dz2[t][j] = ((mask2 >> j) & 1u) ? dout * w3[j] : 0.f;
    for (int i = 0; i < H; ++i) {
        float dh = 0.f;
#pragma unroll
        for (int j = 0; j < H; ++j) dh = fmaf(s_dz2[t][j], w2[j * H + i], dh);
        s_dz1[t][i] = ((mask1 >> i) & 1u) ? dh : 0.f;
    }
    __syncthreads();
    // per-block gradient sums, fixed summation order over the block's samples
    float *g = partial + (size_t)blockIdx.x * kParams;
    for (int e = t; e < H * H; e += kTrainThreads) {  // dL/dw2[j][i] = sum_s dz2[s][j] h1[s][i]
        const int j = e / H, i = e % H;
        float acc = 0.f;
        for (int s2 = 0; s2 < kTrainThreads; ++s2) acc = fmaf(s_dz2[s2][j], s_h1[s2][i], acc);
        g[2 * H + e] = acc;
    }
    if (t < H) {
        float gw1 = 0.f, gb1 = 0.f, gb2 = 0.f, gw3 = 0.f;
        for (int s2 = 0; s2 < kTrainThreads; ++s2) {
            gw1 = fmaf(s_dz1[s2][t], s_x[s2], gw1);
            gb1 += s_dz1[s2][t];
            gb2 += s_dz2[s2][t];
            gw3 = fmaf(s_dout[s2], s_h2[s2][t], gw3);
        }
        g[t] = gw1;
        g[H + t] = gb1;
        g[2 * H + H * H + t] = gb2;
        g[3 * H + H * H + t] = gw3;
    }
    if (t == 0) {
        float gb3 = 0.f, l = 0.f;
        for (int s2 = 0; s2 < kTrainThreads; ++s2) {
            gb3 += s_dout[s2];
            l += s_loss[s2];
        }
        g[4 * H + H * H] = gb3;
        loss_partial[blockIdx.x] = l;
    }
}

// Sums the per-block partials in block order (deterministic): grad[k], loss.
__global__ void rmi_reduce_kernel(const float *__restrict__ partial, const float *__restrict__ loss_partial,
                                  uint32_t blocks, float *__restrict__ grad, float *__restrict__ loss) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < kParams + 1; k += gridDim.x * blockDim.x) {
        float acc = 0.f;
        if (k < kParams)
            for (uint32_t b = 0; b < blocks; ++b) acc += partial[(size_t)b * kParams + k];
        else
            for (uint32_t b = 0; b < blocks; ++b) acc += loss_partial[b];
        if (k < kParams) grad[k] = acc; else *loss = acc;
    }
}

// Adam (Kingma & Ba, ICLR 2015) on the flat parameter vector.
// With `monotone`, the weights of the three layers are projected onto w >= 0
// after each step, which keeps the root non-decreasing in the key (biases stay
// free): every segment then receives one contiguous key range.
__device__ __forceinline__ bool is_weight(int k) {
    return k < H || (k >= 2 * H && k < 2 * H + H * H) || (k >= 3 * H + H * H && k < 4 * H + H * H);
}

__global__ void rmi_adam_kernel(float *__restrict__ w, float *__restrict__ mom, float *__restrict__ vel,
                                const float *__restrict__ grad, float lr, float b1, float b2, float eps,
                                float c1, float c2, int monotone) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < kParams; k += gridDim.x * blockDim.x) {
        const float g = grad[k];
        mom[k] = b1 * mom[k] + (1.f - b1) * g;
        vel[k] = b2 * vel[k] + (1.f - b2) * g * g;
        float nw = w[k] - lr * (mom[k] / c1) / (sqrtf(vel[k] / c2) + eps);
        if (monotone && is_weight(k)) nw = fmaxf(nw, 0.f);
        w[k] = nw;
    }
}

// ---------------------------------------------------------------- leaves
// Each thread walks a contiguous run of sorted keys and emits one set of
// atomics per change of leaf (the root is close to monotone, so runs are long).
constexpr int kLeafChunk = 64;

__global__ void leaf_extent_kernel(const __grid_constant__ ModelParams p, bool use_net, const uint64_t *__restrict__ keys,
                                   uint64_t n, unsigned long long *kmin, unsigned long long *kmax,
                                   unsigned long long *rmin, unsigned long long *rmax) {
    __shared__ PiecesSmem sp;
    if (use_net) stage_pieces(p, sp);
    const uint64_t nthr = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t c = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; c * kLeafChunk < n; c += nthr) {
        const uint64_t s0 = c * kLeafChunk, s1 = min(n, s0 + kLeafChunk);
        uint32_t cur = 0xFFFFFFFFu;
        uint64_t lo_k = 0, hi_k = 0, lo_r = 0, hi_r = 0;
        for (uint64_t s = s0; s <= s1; ++s) {
            uint32_t l = 0xFFFFFFFFu;
            uint64_t k = 0;
            if (s < s1) {
                k = keys[s];
                l = leaf_of(p, root_eval(p, sp, feature(p, k), use_net));
            }
            if (l != cur) {
                if (cur != 0xFFFFFFFFu) {
                    atomicMin(&kmin[cur], (unsigned long long)lo_k);
                    atomicMax(&kmax[cur], (unsigned long long)hi_k);
                    atomicMin(&rmin[cur], (unsigned long long)lo_r);
                    atomicMax(&rmax[cur], (unsigned long long)hi_r);
                }
                cur = l;
                lo_k = hi_k = k;
                lo_r = hi_r = s;
            } else {
                lo_k = min(lo_k, k);
                hi_k = max(hi_k, k);
                lo_r = min(lo_r, s);
                hi_r = max(hi_r, s);
            }
        }
    }
}

// Linear segment through the extreme (key, rank) points of the segment's keys.
__global__ void leaf_fit_kernel(uint32_t L, const unsigned long long *kmin, const unsigned long long *kmax,
                                const unsigned long long *rmin, const unsigned long long *rmax,
                                tl_rank_leaf *leaves) {
    for (uint32_t l = blockIdx.x * blockDim.x + threadIdx.x; l < L; l += gridDim.x * blockDim.x) {
        tl_rank_leaf lf;
        lf.eps_lo = lf.eps_hi = 0;
        if (kmin[l] > kmax[l]) {
            lf.kmin = 0;
            lf.base = 0;
            lf.slope = 0.f;
            lf.empty = 1;
        } else {
            lf.kmin = kmin[l];
            lf.base = rmin[l];
            const double dk = (double)(kmax[l] - kmin[l]);
            lf.slope = dk > 0 ? (float)((double)(rmax[l] - rmin[l]) / dk) : 0.f;
            lf.empty = 0;
        }
        leaves[l] = lf;
    }
}

// An empty segment's window: the ranks from the largest rank of the nearest
// segment below that holds keys to the smallest of the nearest one above
// (where the root is non-decreasing, a query mapped to the empty segment lies
// between those two keys), as base = the lower, slope 0, eps_hi = the span.
// One block of 1024 threads, a contiguous run of segments each; a run's
// nearest holder below and above comes from the runs' summaries.
__global__ void __launch_bounds__(1024) leaf_fill_empty_kernel(uint32_t L, uint64_t n,
                                                               const unsigned long long *__restrict__ rmin,
                                                               const unsigned long long *__restrict__ rmax,
                                                               tl_rank_leaf *__restrict__ leaves) {
    constexpr unsigned long long kNone = ~0ull;
    __shared__ unsigned long long s_last[1024], s_first[1024];
    const uint32_t per = (L + 1023) / 1024, l0 = min(L, threadIdx.x * per), l1 = min(L, l0 + per);
    unsigned long long last = kNone, first = kNone;  // this run's last rmax and first rmin of a holder
    for (uint32_t l = l0; l < l1; ++l)
        if (rmin[l] <= rmax[l]) {
            if (first == kNone) first = rmin[l];
            last = rmax[l];
        }
    s_last[threadIdx.x] = last;
    s_first[threadIdx.x] = first;
    __syncthreads();
    if (threadIdx.x == 0) {  // nearest holder before each run / after each run
        unsigned long long run = kNone;
        for (int t = 0; t < 1024; ++t) {
            const unsigned long long v = s_last[t];
            s_last[t] = run;
            if (v != kNone) run = v;
        }
        run = kNone;
        for (int t = 1023; t >= 0; --t) {
            const unsigned long long v = s_first[t];
            s_first[t] = run;
            if (v != kNone) run = v;
        }
    }
    __syncthreads();
    unsigned long long below = s_last[threadIdx.x];
    for (uint32_t l = l0; l < l1; ++l) {  // the lower end into base
        if (rmin[l] <= rmax[l]) below = rmax[l];
        else leaves[l].base = below;
    }
    unsigned long long above = s_first[threadIdx.x];
    for (uint32_t l = l1; l-- > l0;) {
        if (rmin[l] <= rmax[l]) {
            above = rmin[l];
            continue;
        }
        const uint64_t lo0 = leaves[l].base == kNone ? 0 : leaves[l].base;
        const uint64_t hi0 = above == kNone ? n - 1 : above;
        const uint64_t lo = min(lo0, hi0), hi = max(lo0, hi0);  // a non-monotone root may swap them
        leaves[l].base = lo;
        leaves[l].kmin = 0;
        leaves[l].slope = 0.f;
        leaves[l].eps_lo = 0;
        leaves[l].eps_hi = hi - lo > 0xFFFFFFFEull ? 0xFFFFFFFEu : (uint32_t)(hi - lo);
    }
}

// The segment's error bounds: the largest over- and under-prediction over its
// keys, computed with the inference arithmetic itself.
__global__ void leaf_eps_kernel(const __grid_constant__ ModelParams p, bool use_net, const uint64_t *__restrict__ keys, uint64_t n,
                                tl_rank_leaf *leaves) {
    __shared__ PiecesSmem sp;
    if (use_net) stage_pieces(p, sp);
    const uint64_t nthr = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t c = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; c * kLeafChunk < n; c += nthr) {
        const uint64_t s0 = c * kLeafChunk, s1 = min(n, s0 + kLeafChunk);
        uint32_t cur = 0xFFFFFFFFu, over = 0, under = 0;
        for (uint64_t s = s0; s <= s1; ++s) {
            uint32_t l = 0xFFFFFFFFu, eo = 0, eu = 0;
            if (s < s1) {
                const uint64_t k = keys[s];
                l = leaf_of(p, root_eval(p, sp, feature(p, k), use_net));
                const uint64_t pr = leaf_predict(leaves[l], k, n);
                const uint64_t d = pr > s ? pr - s : s - pr;
                const uint32_t e = d > 0xFFFFFFFEull ? 0xFFFFFFFEu : (uint32_t)d;
                if (pr > s) eo = e; else eu = e;
            }
            if (l != cur) {
                if (cur != 0xFFFFFFFFu) {
                    atomicMax(&leaves[cur].eps_lo, over);
                    atomicMax(&leaves[cur].eps_hi, under);
                }
                cur = l;
                over = eo;
                under = eu;
            } else {
                over = max(over, eo);
                under = max(under, eu);
            }
        }
    }
}

__global__ void rmi_predict_kernel(const __grid_constant__ ModelParams p, bool use_net, const tl_rank_leaf *__restrict__ leaves,
                                   const uint64_t *__restrict__ keys, uint64_t nq, uint64_t n,
                                   uint64_t *__restrict__ rank, uint32_t *__restrict__ eps) {
    __shared__ PiecesSmem sp;
    if (use_net) stage_pieces(p, sp);
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nq;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t k = keys[i];
        const uint32_t l = leaf_of(p, root_eval(p, sp, feature(p, k), use_net));
        const tl_rank_leaf lf = leaves[l];
        rank[i] = leaf_predict(lf, k, n);
        if (eps) eps[i] = lf.empty ? 0xFFFFFFFFu : max(lf.eps_lo, lf.eps_hi);
    }
}

// ---------------------------------------------------------------- learned query
struct LearnedGeom {
    BtreeGeom g;
    FastDiv64 fd;
    uint64_t cmax;  // (n + 1) / (b + 1): nodes below it have a child inside the layout
};

// In-order "gap" coordinates: the top tree's ni keys split the key space into
// ni + 1 gaps; gap j holds leaf node j of the last level (if it exists).  A
// subtree rooted at depth k, index x spans gaps [x S_k, (x+1) S_k - 1] with
// S_k = (b+1)^(h-k).  lower/upper gap of sorted rank s:
__device__ __forceinline__ void rank_gaps(const LearnedGeom &G, uint64_t s, uint64_t &lo, uint64_t &hi) {
    const BtreeGeom &g = G.g;
    if (s < g.l + g.i) {
        uint64_t j, t;
        G.fd.divmod(s, j, t);
        lo = j;
        hi = t < g.b ? j : j + 1;
    } else if (s < g.lir) {
        lo = hi = g.i;
    } else {
        lo = s - g.l - g.r;
        hi = lo + 1;
    }
}

// A node of B = NB / 8 keys (NB = b * 8 bytes): lt = keys < q, eq = a key == q,
// valid = keys below n.  Full nodes by NB / VB independent VB-byte loads (VB =
// 32 on a 32-byte aligned layout, else 16), the partial last leaf by guarded
// scalar loads.
template <int NB, int VB>
__device__ __forceinline__ void node_scan(const uint64_t *__restrict__ A, uint64_t n, uint64_t i, uint64_t q,
                                          uint32_t &lt, uint32_t &valid, bool &eq) {
    constexpr int B = NB / 8, KPL = VB / 8, NL = NB / VB;
    lt = 0;
    eq = false;
    if (i + B <= n) {
        valid = B;
        uint64_t v[NL][32 / 8];
#pragma unroll
        for (int j = 0; j < NL; ++j) {
            if constexpr (VB == 32) {
                ldg32(A + i + j * KPL, v[j]);
            } else {
                const uint4 x = __ldg(reinterpret_cast<const uint4 *>(A + i + j * KPL));
                v[j][0] = ((uint64_t)x.y << 32) | x.x;
                v[j][1] = ((uint64_t)x.w << 32) | x.z;
            }
        }
#pragma unroll
        for (int j = 0; j < NL; ++j)
#pragma unroll
            for (int e = 0; e < KPL; ++e) {
                lt += v[j][e] < q;
                eq |= v[j][e] == q;
            }
    } else {
        valid = (uint32_t)(n - i);
        for (uint32_t j = 0; j < valid; ++j) {
            const uint64_t cur = __ldg(A + i + j);
            lt += cur < q;
            eq |= cur == q;
        }
    }
}

// The start of one query's descent: the deepest subtree whose in-order rank
// range covers the model's window (flags kSubtree), or the root.
constexpr uint32_t kSubtree = 1, kSeenLess = 2, kSeenGreater = 4;

// The segment the rank model's root assigns to q.
__device__ __forceinline__ uint32_t learned_segment(const ModelParams &p, const PiecesSmem &sp, int use_net,
                                                    uint64_t q) {
    return leaf_of(p, root_eval(p, sp, feature(p, q), use_net != 0));
}

template <uint64_t B>
__device__ __forceinline__ uint64_t learned_start_at(const LearnedGeom &G, const tl_rank_leaf &lf, uint64_t q,
                                                     uint32_t &flags, uint32_t &depth) {
    const BtreeGeom &g = G.g;
    const uint64_t n = g.n;
    flags = 0;
    depth = 0;
    if (g.h == 0) return 0;
    const uint64_t pr = leaf_predict(lf, q, n);
    const uint64_t rlo = pr > lf.eps_lo ? pr - lf.eps_lo : 0;
    const uint64_t rhi = pr + lf.eps_hi < n ? pr + lf.eps_hi : n - 1;
    uint64_t glo, ghi, t0, t1;
    rank_gaps(G, rlo, glo, t0);
    rank_gaps(G, rhi, t1, ghi);
    uint32_t k = g.h;  // depth of the subtree root (h = a last-level node)
    while (glo != ghi) {
        glo = G.fd.div(glo);
        ghi = G.fd.div(ghi);
        --k;
    }
    // a last-level node that does not exist: start one level up
    if (k == g.h && !(glo < g.i || (glo == g.i && g.r > 0))) {
        glo = G.fd.div(glo);
        --k;
    }
    const uint64_t i = g.pw[k] - 1 + glo * B;
    if (i >= n) return 0;
    flags = kSubtree;
    depth = k;
    return i;
}

template <uint64_t B>
__device__ __forceinline__ uint64_t learned_start(const LearnedGeom &G, const ModelParams &p, const PiecesSmem &sp,
                                                  int use_net, const tl_rank_leaf *__restrict__ leaves, bool leaves32,
                                                  uint64_t q, uint32_t &flags, uint32_t &depth) {
    const tl_rank_leaf lf = load_leaf(leaves, learned_segment(p, sp, use_net, q), leaves32);
    return learned_start_at<B>(G, lf, q, flags, depth);
}

constexpr uint64_t kIdle = ~0ull;

// 1024-thread blocks: two per SM hold the pieces twice in shared memory (about
// 30 KB), leaving the rest of the unified L1 to the descents' top levels (with
// 256-thread blocks, eight copies took 143 KB of it and the descent slowed by
// a quarter).
#ifndef TL_LEARNED_THREADS
#define TL_LEARNED_THREADS 1024
#endif
#ifndef TL_LEARNED_MIN_BLOCKS
#define TL_LEARNED_MIN_BLOCKS 1
#endif

constexpr int kLearnedThreads = TL_LEARNED_THREADS;
// The group-read kernel: 768-thread blocks, two per SM at 40 registers (no
// spills); measured on B200 (2^28 Zipf queries over 2^30 skewed u64 keys,
// b = 16) 16.4e9 q/s against 15.8e9 with one 1024-thread block per SM, 15.9e9
// with two, 15.6e9 with three 512-thread blocks.
#ifndef TL_LEARNED_GROUP_THREADS
#define TL_LEARNED_GROUP_THREADS 768
#endif
#ifndef TL_LEARNED_GROUP_MIN_BLOCKS
#define TL_LEARNED_GROUP_MIN_BLOCKS 2
#endif
constexpr int kLearnedGroupThreads = TL_LEARNED_GROUP_THREADS;

// One descent per lane, fed from a per-warp queue: a lane whose descent ends
// takes the next prepared query at once, so start depths that differ, hits at
// inner levels and the restarts from the root do not hold the warp's other
// lanes (one query per lane at a time kept 12 of 32 lanes busy on average).
// The queue holds 32 prepared starts, one per lane, computed together when it
// runs dry (the rank model, the window and the start subtree, all lanes busy);
// idle lanes take them in lane order by shuffle.  A descent started below the
// root accepts a miss only when it saw node keys on both sides of the query
// (kSeenLess, kSeenGreater); otherwise it restarts at the root.  Each warp
// answers a contiguous range of the queries.
template <int NB, int VB>
__global__ void __launch_bounds__(kLearnedThreads, TL_LEARNED_MIN_BLOCKS)
learned_query_kernel(const uint64_t *__restrict__ A, const LearnedGeom G, const __grid_constant__ ModelParams p,
                     int use_net, const tl_rank_leaf *__restrict__ leaves, const uint64_t *__restrict__ Q,
                     uint64_t nq, uint64_t *__restrict__ ans, unsigned long long *__restrict__ stats) {
    constexpr uint64_t B = NB / 8;
    // a descent's node index with its flags in the top bits (n < 2^61)
    constexpr uint64_t kFlagShift = 61, kNodeMask = (1ull << kFlagShift) - 1;
    __shared__ PiecesSmem sp;
    if (use_net) stage_pieces(p, sp);
    const bool leaves32 = (reinterpret_cast<uintptr_t>(leaves) & 31) == 0;
    const uint64_t n = G.g.n;
    const uint64_t cmax = (n + 1) / (B + 1);
    const uint32_t lane = threadIdx.x & 31;
    const unsigned below = (1u << lane) - 1u;
    const uint64_t warps = (uint64_t)gridDim.x * (blockDim.x >> 5);
    const uint64_t w = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint64_t per = (nq + warps - 1) / warps;  // below 2^32 (the host checks q)
    const uint64_t q0 = min(nq, w * per);
    const uint32_t cnt = (uint32_t)(min(nq, q0 + per) - q0);  // the warp's queries: q0 .. q0 + cnt
    uint32_t n_fallback = 0, depth_sum = 0;
    uint64_t cur = kIdle, key = 0;  // this lane's descent: node | flags << kFlagShift
    uint32_t qoff = 0;
    uint64_t e_cur = 0, e_key = 0;  // this lane's prepared entry of the current batch
    uint32_t next = 0, batch0 = 0, bn = 0, bpos = 0;
    for (;;) {
        unsigned need = __ballot_sync(0xFFFFFFFFu, cur == kIdle);
        while (need) {
            if (bpos == bn) {
                if (next >= cnt) break;
                batch0 = next;
                bn = cnt - next < 32 ? cnt - next : 32;
                bpos = 0;
                next += bn;
                if (lane < bn) {
                    e_key = __ldcs(Q + q0 + batch0 + lane);
                    uint32_t f, d;
                    const uint64_t nd = learned_start<B>(G, p, sp, use_net, leaves, leaves32, e_key, f, d);
                    e_cur = nd | ((uint64_t)f << kFlagShift);
                    if (f) depth_sum += d; else ++n_fallback;
                }
            }
            const uint32_t avail = bn - bpos;
            unsigned take = need;
            if ((uint32_t)__popc(need) > avail) {  // the lowest `avail` idle lanes
                take = 0;
                unsigned m = need;
                for (uint32_t c = 0; c < avail; ++c) {
                    const unsigned low = m & (0u - m);
                    take |= low;
                    m ^= low;
                }
            }
            const bool mine = (take >> lane) & 1u;
            const uint32_t src = bpos + __popc(take & below);
            const uint64_t k2 = __shfl_sync(0xFFFFFFFFu, e_key, mine ? src : 0);
            const uint64_t c2 = __shfl_sync(0xFFFFFFFFu, e_cur, mine ? src : 0);
            if (mine) {
                key = k2;
                cur = c2;
                qoff = batch0 + src;
            }
            bpos += __popc(take);
            need &= ~take;
        }
        if (!__any_sync(0xFFFFFFFFu, cur != kIdle)) break;
        if (cur != kIdle) {
            const uint64_t node = cur & kNodeMask;
            uint32_t fl = (uint32_t)(cur >> kFlagShift);
            uint32_t lt, valid;
            bool eq;
            node_scan<NB, VB>(A, n, node, key, lt, valid, eq);
            uint64_t res = kIdle;
            if (eq) {
                res = node + lt;
            } else {
                fl |= (lt > 0 ? kSeenLess : 0u) | (lt < valid ? kSeenGreater : 0u);
                const uint64_t nx = node + 1 <= cmax ? (node + 1) * (B + 1) + (uint64_t)lt * B - 1 : n;
                if (nx < n) {
                    cur = nx | ((uint64_t)fl << kFlagShift);
                } else if (!(fl & kSubtree) || ((fl & kSeenLess) && (fl & kSeenGreater))) {
                    res = n;  // absent (from the root; or the subtree straddles the query)
                } else {      // the window could not decide: plain search from the root
                    ++n_fallback;
                    cur = 0;
                }
            }
            if (res != kIdle) {
                __stcs(ans + q0 + qoff, res);
                cur = kIdle;
            }
        }
    }
    if (stats) {
        unsigned long long f = n_fallback, d = depth_sum;
        for (int o = 16; o > 0; o >>= 1) {
            f += __shfl_xor_sync(0xFFFFFFFFu, f, o);
            d += __shfl_xor_sync(0xFFFFFFFFu, d, o);
        }
        if ((threadIdx.x & 31) == 0) {
            atomicAdd(&stats[0], f);
            atomicAdd(&stats[1], d);
        }
    }
}

// ---------------------------------------------------------------- host
// The same queue feeding a group of GL lanes per descent instead of one lane:
// lane g reads node slots 4g + 4 GL j + [0, 4) with load j of NL = NB / (32 GL)
// 32-byte loads, so each load instruction of a warp touches 32 / GL node lines
// of GL sectors, one L1 wavefront each (the plain B-tree query's node read).
// Idle groups take the prepared starts in group order; the group adds its
// lanes' counts with full-warp shuffles and learns of an equal key by ballot.
template <int NB, int GL, bool kStats>
__global__ void __launch_bounds__(kLearnedGroupThreads, TL_LEARNED_GROUP_MIN_BLOCKS)
learned_query_group_kernel(const uint64_t *__restrict__ A, const LearnedGeom G, const __grid_constant__ ModelParams p,
                           int use_net, const tl_rank_leaf *__restrict__ leaves, const uint64_t *__restrict__ Q,
                           uint64_t nq, uint64_t *__restrict__ ans, unsigned long long *__restrict__ stats) {
    constexpr uint64_t B = NB / 8;
    constexpr int KPL = 4;               // keys per 32-byte load
    constexpr int NL = NB / (32 * GL);   // loads per lane and node
    static_assert((GL == 2 || GL == 4 || GL == 8) && NL >= 1 && NL * GL * 32 == NB, "2, 4 or 8 lanes per node");
    constexpr unsigned kLeaders = GL == 2 ? 0x55555555u : GL == 4 ? 0x11111111u : 0x01010101u;
    constexpr uint64_t kFlagShift = 61, kNodeMask = (1ull << kFlagShift) - 1;
    __shared__ PiecesSmem sp;
    if (use_net) stage_pieces(p, sp);
    const bool leaves32 = (reinterpret_cast<uintptr_t>(leaves) & 31) == 0;
    const uint64_t n = G.g.n;
    const uint64_t cmax = G.cmax;
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t g = lane % GL, lead = lane - g;
    const unsigned below = (1u << lane) - 1u, below_lead = (1u << lead) - 1u;
    const uint64_t warps = (uint64_t)gridDim.x * (blockDim.x >> 5);
    const uint64_t w = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint64_t per = (nq + warps - 1) / warps;  // below 2^32 (the host checks q)
    const uint64_t q0 = min(nq, w * per);
    const uint32_t cnt = (uint32_t)(min(nq, q0 + per) - q0);
    uint32_t n_fallback = 0, depth_sum = 0;
    uint64_t cur = kIdle, key = 0;  // this group's descent: node | flags << kFlagShift
    uint32_t qoff = 0;
    uint64_t e_cur = 0, e_key = 0;  // this lane's prepared entry of the current batch
    uint32_t next = 0, batch0 = 0, bn = 0, bpos = 0;
    (void)below;
    for (;;) {
        unsigned need = __ballot_sync(0xFFFFFFFFu, cur == kIdle) & kLeaders;
        while (need) {
            if (bpos == bn) {
                if (next >= cnt) break;
                batch0 = next;
                bn = cnt - next < 32 ? cnt - next : 32;
                bpos = 0;
                next += bn;
                if (lane < bn) {
                    e_key = __ldcs(Q + q0 + batch0 + lane);
                    uint32_t f, d;
                    const uint64_t nd = learned_start<B>(G, p, sp, use_net, leaves, leaves32, e_key, f, d);
                    e_cur = nd | ((uint64_t)f << kFlagShift);
                    if (kStats) {
                        if (f) depth_sum += d; else ++n_fallback;
                    }
                }
            }
            const uint32_t avail = bn - bpos;
            unsigned take = need;
            if ((uint32_t)__popc(need) > avail) {  // the lowest `avail` idle groups
                take = 0;
                unsigned m = need;
                for (uint32_t c = 0; c < avail; ++c) {
                    const unsigned low = m & (0u - m);
                    take |= low;
                    m ^= low;
                }
            }
            const bool mine = (take >> lead) & 1u;
            const uint32_t src = bpos + __popc(take & below_lead);
            const uint64_t k2 = __shfl_sync(0xFFFFFFFFu, e_key, mine ? src : 0);
            const uint64_t c2 = __shfl_sync(0xFFFFFFFFu, e_cur, mine ? src : 0);
            if (mine) {
                key = k2;
                cur = c2;
                qoff = batch0 + src;
            }
            bpos += __popc(take);
            need &= ~take;
        }
        if (!__any_sync(0xFFFFFFFFu, cur != kIdle)) break;
        const bool live = cur != kIdle;
        const uint64_t node = cur & kNodeMask;
        uint32_t lt = 0;
        bool eq = false;
        if (live) {
            const uint64_t s0 = node + (uint64_t)g * KPL;
            if (node + B <= n) {
                uint64_t v[NL][KPL];
#pragma unroll
                for (int j = 0; j < NL; ++j) ldg32(A + s0 + (uint64_t)j * GL * KPL, v[j]);
#pragma unroll
                for (int j = 0; j < NL; ++j)
#pragma unroll
                    for (int e = 0; e < KPL; ++e) {
                        lt += v[j][e] < key;
                        eq |= v[j][e] == key;
                    }
            } else {  // the partial last leaf: slots at or past n do not count
#pragma unroll
                for (int j = 0; j < NL; ++j)
#pragma unroll
                    for (int e = 0; e < KPL; ++e) {
                        const uint64_t pos = s0 + (uint64_t)j * GL * KPL + e;
                        if (pos < n) {
                            const uint64_t c = __ldg(A + pos);
                            lt += c < key;
                            eq |= c == key;
                        }
                    }
            }
        }
#pragma unroll
        for (int off = GL / 2; off > 0; off >>= 1) lt += __shfl_xor_sync(0xFFFFFFFFu, lt, off);
        const bool hit = ((__ballot_sync(0xFFFFFFFFu, eq) >> lead) & ((1u << GL) - 1)) != 0;
        if (live) {
            const uint32_t valid = node + B <= n ? (uint32_t)B : (uint32_t)(n - node);
            uint32_t fl = (uint32_t)(cur >> kFlagShift);
            uint64_t res = kIdle;
            if (hit) {
                res = node + lt;
            } else {
                fl |= (lt > 0 ? kSeenLess : 0u) | (lt < valid ? kSeenGreater : 0u);
                const uint64_t nx = node + 1 <= cmax ? (node + 1) * (B + 1) + (uint64_t)lt * B - 1 : n;
                if (nx < n) {
                    cur = nx | ((uint64_t)fl << kFlagShift);
                } else if (!(fl & kSubtree) || ((fl & kSeenLess) && (fl & kSeenGreater))) {
                    res = n;  // absent (from the root; or the subtree straddles the query)
                } else {      // the window could not decide: plain search from the root
                    if (kStats && g == 0) ++n_fallback;
                    cur = 0;
                }
            }
            if (res != kIdle) {
                if (g == 0) __stcs(ans + q0 + qoff, res);
                cur = kIdle;
            }
        }
    }
    if (kStats && stats) {
        unsigned long long f = n_fallback, d = depth_sum;
        for (int o = 16; o > 0; o >>= 1) {
            f += __shfl_xor_sync(0xFFFFFFFFu, f, o);
            d += __shfl_xor_sync(0xFFFFFFFFu, d, o);
        }
        if ((threadIdx.x & 31) == 0) {
            atomicAdd(&stats[0], f);
            atomicAdd(&stats[1], d);
        }
    }
}

static void init_model(tl_rank_model &m, const tl_rank_train_config &cfg) {
    memset(&m, 0, sizeof m);
    // layer 1: ramps with breakpoints spread over [0, 1]
    for (int i = 0; i < H; ++i) {
        m.w1[i] = 1.f;
        m.b1[i] = -(float)i / H;
    }
    // layer 2: small deterministic pseudo-random weights
    for (int j = 0; j < H; ++j) {
        for (int i = 0; i < H; ++i) {
            uint64_t r = mix64(cfg.seed * 1315423911ull + (uint64_t)(j * H + i));
            m.w2[j][i] = ((float)(r >> 40) / (float)(1u << 24) - 0.5f) * (2.f / H);
            if (cfg.monotone) m.w2[j][i] = fabsf(m.w2[j][i]);
        }
        m.b2[j] = 0.01f;
        m.w3[j] = 1.f / H;
    }
    m.b3 = 0.f;
}

static void model_to_flat(const tl_rank_model &m, float *w) {
    memcpy(w, m.w1, sizeof m.w1);
    memcpy(w + H, m.b1, sizeof m.b1);
    memcpy(w + 2 * H, m.w2, sizeof m.w2);
    memcpy(w + 2 * H + H * H, m.b2, sizeof m.b2);
    memcpy(w + 3 * H + H * H, m.w3, sizeof m.w3);
    w[4 * H + H * H] = m.b3;
}

static void flat_to_model(const float *w, tl_rank_model &m) {
    memcpy(m.w1, w, sizeof m.w1);
    memcpy(m.b1, w + H, sizeof m.b1);
    memcpy(m.w2, w + 2 * H, sizeof m.w2);
    memcpy(m.b2, w + 2 * H + H * H, sizeof m.b2);
    memcpy(m.w3, w + 3 * H + H * H, sizeof m.w3);
    m.b3 = w[4 * H + H * H];
}

static int grid_for(uint64_t work, int threads) {
    uint64_t g = (work + threads - 1) / threads;
    return (int)std::max<uint64_t>(1, std::min<uint64_t>(g, 148ull * 16));
}

static Feature feature_params(const tl_rank_model &m) {
    Feature f;
    f.x_lo = (float)m.x_lo;
    f.x_scale = (float)m.x_scale;
    f.log_feature = m.log_feature;
    return f;
}

int rank_model_gradient(const tl_rank_model *m, const float *dx, const float *dy, uint32_t count, float *grad,
                        float *loss, cudaStream_t st) {
    if (!m || !dx || !dy || !grad || count == 0) return TL_ERROR_INVALID_VALUE;
    const uint32_t blocks = (count + kTrainThreads - 1) / kTrainThreads;
    float *buf = nullptr;
    const size_t bytes = ((size_t)blocks * kParams + blocks + 2 * (kParams + 1)) * sizeof(float);
    keep_pool_memory();
    TL_CUDA_TRY(cudaMallocAsync(reinterpret_cast<void **>(&buf), bytes, st));
    float *partial = buf, *lp = buf + (size_t)blocks * kParams, *g = lp + blocks, *w = g + kParams + 1;
    float flat[kParams + 1] = {0};
    model_to_flat(*m, flat);
    cudaError_t e = cudaMemcpyAsync(w, flat, kParams * sizeof(float), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
        rmi_grad_kernel<<<blocks, kTrainThreads, 0, st>>>(w, feature_params(*m), dx, dy, nullptr, 1, 0, count,
                                                          1.f / count, partial, lp);
        rmi_reduce_kernel<<<8, 256, 0, st>>>(partial, lp, blocks, g, g + kParams);
        e = cudaGetLastError();
    }
    float host[kParams + 1];
    if (e == cudaSuccess) e = cudaMemcpyAsync(host, g, sizeof host, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFreeAsync(buf, st);
    if (e != cudaSuccess) {
        record_cuda_error(e);
        return TL_ERROR_CUDA;
    }
    memcpy(grad, host, kParams * sizeof(float));
    if (loss) *loss = host[kParams];
    return TL_SUCCESS;
}

int rank_model_train(const uint64_t *keys, uint64_t n, const tl_rank_train_config *cfg, tl_rank_model *out,
                     tl_rank_leaf *leaves, cudaStream_t st) {
    if (!keys || !cfg || !out || !leaves || n < 2) return TL_ERROR_INVALID_VALUE;
    const uint32_t L = cfg->num_leaves;
    if (L == 0 || (L & (L - 1)) || L > (1u << 24)) return TL_ERROR_INVALID_VALUE;
    tl_rank_model m;
    init_model(m, *cfg);
    m.num_leaves = L;
    m.log_feature = cfg->log_feature;
    m.n = n;
    uint64_t kfirst = 0, klast = 0;
    TL_CUDA_TRY(cudaMemcpyAsync(&kfirst, keys, 8, cudaMemcpyDeviceToHost, st));
    TL_CUDA_TRY(cudaMemcpyAsync(&klast, keys + n - 1, 8, cudaMemcpyDeviceToHost, st));
    TL_CUDA_TRY(cudaStreamSynchronize(st));
    const double f0 = m.log_feature ? (double)std::log2((float)kfirst + 1.0f) : (double)kfirst;
    const double f1 = m.log_feature ? (double)std::log2((float)klast + 1.0f) : (double)klast;
    m.x_lo = f0;
    m.x_scale = f1 > f0 ? 1.0 / (f1 - f0) : 1.0;
    const Feature fe = feature_params(m);

    const uint32_t batch = std::max<uint32_t>(kTrainThreads, cfg->batch);
    const uint32_t blocks = (batch + kTrainThreads - 1) / kTrainThreads;
    float *buf = nullptr;
    const size_t nfl = (size_t)blocks * kParams + blocks + 4 * (kParams + 1);
    unsigned long long *ext = nullptr;
    keep_pool_memory();
    TL_CUDA_TRY(cudaMallocAsync(reinterpret_cast<void **>(&buf), nfl * sizeof(float), st));
    TL_CUDA_TRY(cudaMallocAsync(reinterpret_cast<void **>(&ext), 4ull * L * sizeof(unsigned long long), st));
    float *partial = buf, *lp = partial + (size_t)blocks * kParams, *grad = lp + blocks;
    float *w = grad + kParams + 1, *mom = w + kParams + 1, *vel = mom + kParams + 1;
    float flat[kParams + 1] = {0};
    model_to_flat(m, flat);
    TL_CUDA_TRY(cudaMemcpyAsync(w, flat, kParams * sizeof(float), cudaMemcpyHostToDevice, st));
    TL_CUDA_TRY(cudaMemsetAsync(mom, 0, 2 * (kParams + 1) * sizeof(float), st));
    const bool use_net = cfg->train_root != 0;
    if (use_net) {
        const float b1 = 0.9f, b2 = 0.999f;
        float c1 = 1.f, c2 = 1.f;
        for (uint32_t step = 0; step < cfg->steps; ++step) {
            rmi_grad_kernel<<<blocks, kTrainThreads, 0, st>>>(w, fe, nullptr, nullptr, keys, n,
                                                              mix64(cfg->seed + step), batch, 1.f / batch,
                                                              partial, lp);
            rmi_reduce_kernel<<<8, 256, 0, st>>>(partial, lp, blocks, grad, grad + kParams);
            c1 *= b1;
            c2 *= b2;
            const float lr = cfg->lr * (step < cfg->steps / 2 ? 1.f : (step < 3 * cfg->steps / 4 ? 0.3f : 0.1f));
            rmi_adam_kernel<<<8, 256, 0, st>>>(w, mom, vel, grad, lr, b1, b2, 1e-8f, 1.f - c1, 1.f - c2,
                                               (int)cfg->monotone);
            TL_CUDA_TRY(cudaGetLastError());
        }
        TL_CUDA_TRY(cudaMemcpyAsync(flat, w, kParams * sizeof(float), cudaMemcpyDeviceToHost, st));
        TL_CUDA_TRY(cudaMemcpyAsync(&m.train_loss, grad + kParams, sizeof(float), cudaMemcpyDeviceToHost, st));
        TL_CUDA_TRY(cudaStreamSynchronize(st));
        flat_to_model(flat, m);
    }
    // leaves
    const ModelParams p = to_params(m);
    unsigned long long *kmin = ext, *kmax = ext + L, *rmin = ext + 2ull * L, *rmax = ext + 3ull * L;
    TL_CUDA_TRY(cudaMemsetAsync(kmin, 0xFF, L * sizeof(unsigned long long), st));
    TL_CUDA_TRY(cudaMemsetAsync(kmax, 0, L * sizeof(unsigned long long), st));
    TL_CUDA_TRY(cudaMemsetAsync(rmin, 0xFF, L * sizeof(unsigned long long), st));
    TL_CUDA_TRY(cudaMemsetAsync(rmax, 0, L * sizeof(unsigned long long), st));
    const uint64_t chunks = (n + kLeafChunk - 1) / kLeafChunk;
    leaf_extent_kernel<<<grid_for(chunks, 256), 256, 0, st>>>(p, use_net, keys, n, kmin, kmax, rmin, rmax);
    leaf_fit_kernel<<<grid_for(L, 256), 256, 0, st>>>(L, kmin, kmax, rmin, rmax, leaves);
    leaf_fill_empty_kernel<<<1, 1024, 0, st>>>(L, n, rmin, rmax, leaves);
    leaf_eps_kernel<<<grid_for(chunks, 256), 256, 0, st>>>(p, use_net, keys, n, leaves);
    TL_CUDA_TRY(cudaGetLastError());
    cudaFreeAsync(buf, st);
    cudaFreeAsync(ext, st);
    TL_CUDA_TRY(cudaStreamSynchronize(st));
    m.train_root = use_net ? 1 : 0;
    *out = m;
    return TL_SUCCESS;
}

int rank_model_root_eval(const tl_rank_model *m, const float *x, uint32_t count, float *out, uint32_t *pieces) {
    if (!m || (count && (!x || !out))) return TL_ERROR_INVALID_VALUE;
    std::unique_ptr<RootPieces> rp(new RootPieces);
    compile_root(*m, *rp);
    for (uint32_t i = 0; i < count; ++i) out[i] = pieces_eval(rp->x0, rp->s, rp->t, rp->first, x[i]);
    if (pieces) *pieces = rp->count;
    return TL_SUCCESS;
}

int rank_model_predict(const tl_rank_model *m, const tl_rank_leaf *leaves, const uint64_t *keys, uint64_t q,
                       uint64_t *rank, uint32_t *eps, cudaStream_t st) {
    if (!m || !leaves || (q && (!keys || !rank))) return TL_ERROR_INVALID_VALUE;
    if (q == 0) return TL_SUCCESS;
    rmi_predict_kernel<<<grid_for(q, 256), 256, 0, st>>>(to_params(*m), m->train_root != 0, leaves, keys, q, m->n,
                                                         rank, eps);
    TL_CUDA_TRY(cudaGetLastError());
    return TL_SUCCESS;
}

int query_btree_learned(const uint64_t *A, uint64_t n, uint64_t b, const tl_rank_model *m,
                        const tl_rank_leaf *leaves, const uint64_t *Q, uint64_t q, uint64_t *ans,
                        unsigned long long *stats, cudaStream_t st, float *ms) {
    if (!m || !leaves || (q && (!Q || !ans)) || (n && !A)) return TL_ERROR_INVALID_VALUE;
    if (m->n != n) return TL_ERROR_INVALID_VALUE;
    // vector node loads: b in {2, 4, 8, 16, 32} on a 16-byte aligned layout
    if (b * 8 % 16 || b * 8 > 256 || ((b * 8 / 16) & (b * 8 / 16 - 1))) return TL_ERROR_UNSUPPORTED;
    if (reinterpret_cast<uintptr_t>(A) & 15) return TL_ERROR_INVALID_VALUE;
    // the kernel keeps a warp's query offsets in 32 bits and a node index with
    // three flag bits in 64
    if (n >= (1ull << 61) || q >= (1ull << 44)) return TL_ERROR_UNSUPPORTED;
    if (q == 0) return TL_SUCCESS;
    LearnedGeom G;
    G.g = make_btree_geom(n, b);
    G.fd = FastDiv64(b + 1);
    G.cmax = (n + 1) / (b + 1);
    EventTimer timer(ms != nullptr, st);
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const ModelParams p = to_params(*m);
    const int use_net = m->train_root != 0;
    auto launch_with = [&](auto kern, int threads) -> int {
        // the smallest shared-memory carve-out that holds the blocks' pieces:
        // the rest stays L1
        TL_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 15));
        int per_sm = 0;
        TL_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, 0));
        uint64_t grid = std::min<uint64_t>((uint64_t)std::max(per_sm, 1) * sms, (q + threads - 1) / threads);
        timer.start();
        kern<<<(unsigned)std::max<uint64_t>(grid, 1), threads, 0, st>>>(A, G, p, use_net, leaves, Q, q, ans, stats);
        return TL_SUCCESS;
    };
    auto launch = [&](auto kern) -> int { return launch_with(kern, kLearnedThreads); };
    auto launch_group = [&](auto kern) -> int { return launch_with(kern, kLearnedGroupThreads); };
    // 64-, 128- and 256-byte nodes on a 32-byte aligned layout: a group of
    // lanes per descent; else one lane per descent with 32-byte node loads
    // (32-byte aligned layout, node bytes a multiple of 32) or 16-byte ones
    const bool v32 = (reinterpret_cast<uintptr_t>(A) & 31) == 0 && (b * 8) % 32 == 0;
    const bool grp = v32 && query_variant() != 6;
    int rc;
    switch (b * 8) {
        case 16: rc = launch(learned_query_kernel<16, 16>); break;
        case 32: rc = v32 ? launch(learned_query_kernel<32, 32>) : launch(learned_query_kernel<32, 16>); break;
        case 64:
            rc = grp   ? (stats ? launch_group(learned_query_group_kernel<64, 2, true>)
                                : launch_group(learned_query_group_kernel<64, 2, false>))
                 : v32 ? launch(learned_query_kernel<64, 32>)
                       : launch(learned_query_kernel<64, 16>);
            break;
        case 128:
            rc = grp && query_variant() == 7
                     ? (stats ? launch_group(learned_query_group_kernel<128, 4, true>)
                              : launch_group(learned_query_group_kernel<128, 4, false>))
                 : grp   ? (stats ? launch_group(learned_query_group_kernel<128, 2, true>)
                                  : launch_group(learned_query_group_kernel<128, 2, false>))
                 : v32 ? launch(learned_query_kernel<128, 32>)
                       : launch(learned_query_kernel<128, 16>);
            break;
        case 256:
            rc = grp   ? (stats ? launch_group(learned_query_group_kernel<256, 4, true>)
                                : launch_group(learned_query_group_kernel<256, 4, false>))
                 : v32 ? launch(learned_query_kernel<256, 32>)
                       : launch(learned_query_kernel<256, 16>);
            break;
        default: return TL_ERROR_UNSUPPORTED;
    }
    if (rc) return rc;
    timer.stop();
    TL_CUDA_TRY(cudaGetLastError());
    if (ms) {
        rc = sync_and_check(st);
        if (rc) return rc;
        *ms = timer.elapsed();
    }
    return TL_SUCCESS;
}

}  // namespace tl
