/*
 * CPU oracle for the tree-layout hot path.  TEST INFRASTRUCTURE ONLY: only the
 * tests, the smoke check and the benchmark's CPU-baseline leg load this file's
 * library.  It restates the reference's algorithms step by step (sequential
 * semantics of each reference kernel); it is not the product.
 *
 * Reference paths cited below are relative to the algoparc/Tree-Layouts tree.
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

/* ------------------------------------------------------------------------ */
/* Array rotations by three reversals: cpu/src/common.h:160-189 (shift_right)  */
/* and cpu/src/common.h:229-258 (shift_left); GPU twins gpu/src/common.cuh:66-110
 * and gpu/src/cycles.cuh:31-236.                                             */
/* ------------------------------------------------------------------------ */
static void rev_swap(uint64_t *A, uint64_t i, uint64_t j) {
    uint64_t t = A[i];
    A[i] = A[j];
    A[j] = t;
}

static void shift_right(uint64_t *A, uint64_t n, uint64_t k) {
    uint64_t i;
    for (i = 0; i < n / 2; ++i) rev_swap(A, i, n - i - 1);
    for (i = 0; i < k / 2; ++i) rev_swap(A, i, k - i - 1);
    for (i = k; i < (n + k) / 2; ++i) rev_swap(A, i, n - (i - k) - 1);
}

static void shift_left(uint64_t *A, uint64_t n, uint64_t k) {
    uint64_t i;
    for (i = 0; i < k / 2; ++i) rev_swap(A, i, k - i - 1);
    for (i = k; i < (n + k) / 2; ++i) rev_swap(A, i, n - (i - k) - 1);
    for (i = 0; i < n / 2; ++i) rev_swap(A, i, n - i - 1);
}

/* ------------------------------------------------------------------------ */
/* Equidistant gather of r roots spaced l+1 apart: cpu/src/cycles.h:31-54     */
/* (GPU phases gpu/src/cycles.cuh:242-287 compute the same permutation).      */
/* ------------------------------------------------------------------------ */
static void equidistant_gather(uint64_t *A, uint64_t r, uint64_t l) {
    for (uint64_t i = 0; i < r; ++i) {
        uint64_t temp = A[(i + 1) * (l + 1) - 1];
        for (uint64_t j = (i + 1) * (l + 1) - 1; j > i; j -= l) A[j] = A[j - l];
        A[i] = temp;
    }
    for (uint64_t i = 0; i < r; ++i) {
        uint64_t kr = r - i;
        uint64_t kl = l - r + i;
        if (kr <= kl && kr != 0 && kr != l)
            shift_right(&A[r + i * l], l, kr);
        else if (kl != 0 && kl != l)
            shift_left(&A[r + i * l], l, kl);
    }
}

/* Chunked equidistant gather: cpu/src/cycles.h:202-239.  The reference moves
 * each chunk of c words through its cycle in sub-blocks of B words; moving the
 * whole chunk at once is the same permutation. */
static void equidistant_gather_chunks(uint64_t *A, uint64_t m, uint64_t c) {
    uint64_t *temp = (uint64_t *)malloc((c ? c : 1) * sizeof(uint64_t));
    for (uint64_t i = 0; i < m; ++i) {
        memcpy(temp, &A[((i + 1) * (m + 1) - 1) * c], c * sizeof(uint64_t));
        for (uint64_t k = ((i + 1) * (m + 1) - 1) * c; k > i * c; k -= m * c)
            memmove(&A[k], &A[k - m * c], c * sizeof(uint64_t));
        memcpy(&A[i * c], temp, c * sizeof(uint64_t));
    }
    free(temp);
    for (uint64_t i = 0; i < m; ++i) {
        uint64_t kr = (m - i) * c;
        uint64_t kl = i * c;
        if (kr <= kl && kr != 0 && kr != m * c)
            shift_right(&A[(i + 1) * m * c], m * c, kr);
        else if (kl != 0 && kl != m * c)
            shift_left(&A[(i + 1) * m * c], m * c, kl);
    }
}

/* Extended equidistant gather, n = (b+1)^d - 1: cpu/src/cycles.h:366-382. */
static void extended_equidistant_gather(uint64_t *A, uint64_t n, uint64_t b) {
    uint64_t m = n / (b + 1);
    if (m <= b) {
        equidistant_gather(A, m, m);
    } else {
        for (uint64_t i = 0; i < b + 1; ++i) extended_equidistant_gather(&A[i * m + i], m, b);
        uint64_t c = (m + b) / (b + 1); /* ceil(m / (b+1)) */
        equidistant_gather_chunks(&A[c - 1], b, c);
    }
}

/* Extended equidistant gather, n = m(b+1): cpu/src/cycles.h:418-445. */
static void extended_equidistant_gather2(uint64_t *A, uint64_t n, uint64_t b) {
    uint64_t m = n / (b + 1);
    if (m <= b) {
        equidistant_gather(A, m, b);
    } else {
        uint64_t r = m % (b + 1);
        if (r == 0) {
            for (uint64_t i = 0; i < b + 1; ++i) extended_equidistant_gather2(&A[i * m], m, b);
            uint64_t c = m / (b + 1);
            equidistant_gather_chunks(&A[c], (m - c) / c, c);
        } else {
            uint64_t size = r * (b + 1);
            extended_equidistant_gather2(A, n - size, b);
            extended_equidistant_gather2(&A[n - size], size, b);
            shift_right(&A[m - r], (m - r) * b + r, r);
        }
    }
}

/* Exact floor(log_{base}(n)) for n >= 1.  The reference computes the level count
 * as log10(n)/log10(b+1) in double (gpu/src/btree-cycles.cuh:81); that agrees with
 * this exact count everywhere the reference's own arithmetic is well defined (at
 * n = (b+1)^k the float form can land one low, after which the reference
 * underflows numInternals - i). */
static uint32_t ilog(uint64_t n, uint64_t base) {
    uint32_t h = 0;
    uint64_t p = 1;
    while (p <= n / base) {
        p *= base;
        ++h;
    }
    return h;
}

static uint64_t ipow(uint64_t base, uint32_t e) {
    uint64_t p = 1;
    while (e--) p *= base;
    return p;
}

/* B-tree permutation: host logic gpu/src/btree-cycles.cuh:77-104 (level count,
 * perfect/non-perfect split, `while (d > 1)` loop of :64-71), leaf handling
 * cpu/src/btree-cycles.h:32-39 (permute_leaves), per-level gathers
 * cpu/src/cycles.h:366-445.  b = 1 is the BST, as gpu/test/build-bst-cycles.cu:39
 * uses it. */
int orc_permute_btree(uint64_t *A, uint64_t n, uint64_t b) {
    if (b == 0) return 1;
    if (n == 0) return 0;
    uint32_t h = ilog(n, b + 1);
    uint32_t d;
    uint64_t nn;
    if (n != ipow(b + 1, h + 1) - 1) {
        uint64_t numInternals = ipow(b + 1, h) - 1;
        uint64_t numLeaves = n - numInternals;
        uint64_t r = numLeaves % b;
        uint64_t l = numLeaves - r;
        uint64_t i = l / b;
        extended_equidistant_gather2(A, l + i, b);
        shift_right(&A[i], numLeaves + numInternals - i, numInternals - i);
        nn = n - numLeaves;
        d = h;
    } else {
        nn = n;
        d = h + 1;
    }
    while (d > 1) {
        extended_equidistant_gather(A, nn, b);
        nn /= b + 1;
        d--;
    }
    return 0;
}

int orc_permute_bst(uint64_t *A, uint64_t n) { return orc_permute_btree(A, n, 1); }

/* ------------------------------------------------------------------------ */
/* Modified van Emde Boas: gpu/src/mveb-cycles.cuh                            */
/* ------------------------------------------------------------------------ */

/* Split of a tree of d levels into a top of root_d and bottoms of leaf_d levels,
 * leaf_d rounded up to a power of two: gpu/src/mveb-cycles.cuh:240-247. */
static void mveb_split(uint32_t d, uint32_t *root_d, uint32_t *leaf_d) {
    uint32_t rd = (d - 2) / 2 + 1;
    uint32_t ld = d - rd;
    float log_leaf = log2f((float)ld);
    if (log_leaf - ((int)log_leaf) != 0) {
        ld = (uint32_t)pow(2, ceil(log_leaf));
        rd = d - ld;
    }
    *root_d = rd;
    *leaf_d = ld;
}

static int is_pow2_levels(uint32_t d) {
    float lg = log2f((float)d);
    return lg - ((int)lg) == 0;
}

/* Sequential semantics of equidistant_gather_warps (gpu/src/cycles.cuh:405-431):
 * the cycles, then always a right rotation of the i-th block by r-i. */
static void equidistant_gather_warps(uint64_t *A, uint64_t r, uint64_t l) {
    for (uint64_t i = 0; i < r; ++i) {
        uint64_t temp = A[(i + 1) * (l + 1) - 1];
        for (uint64_t j = (i + 1) * (l + 1) - 1; j > i; j -= l) A[j] = A[j - l];
        A[i] = temp;
    }
    for (uint64_t i = 0; i < r; ++i)
        if (r - i != 0 && r - i != l) shift_right(&A[r + i * l], l, r - i);
}

/* Base cases: gpu/src/mveb-cycles.cuh:32-112. */
static void basecase2(uint64_t *A, uint64_t n) {
    for (uint64_t i = 0; i < n / 3; ++i) rev_swap(A, 3 * i, 3 * i + 1);
}

static void basecase4(uint64_t *A, uint64_t n) {
    for (uint64_t i = 0; i < n / 15; ++i) {
        uint64_t *a = &A[i * 15];
        equidistant_gather_warps(a, 3, 3);
        for (int t = 0; t < 5; ++t) rev_swap(a, 3 * t, 3 * t + 1);
    }
}

static void basecase8(uint64_t *A, uint64_t n) {
    for (uint64_t i = 0; i < n / 255; ++i) {
        uint64_t *block_a = &A[i * 255];
        equidistant_gather(block_a, 15, 15); /* equidistant_gather_blocks, :375-403 */
        for (int j = 0; j < 17; ++j) {
            uint64_t *warp_a = &block_a[j * 15];
            equidistant_gather_warps(warp_a, 3, 3);
            for (int t = 0; t < 5; ++t) rev_swap(warp_a, 3 * t, 3 * t + 1);
        }
    }
}

/* permutevEB_balanced: gpu/src/mveb-cycles.cuh:118-228.  Each grid-level round
 * gathers sqrt(m) roots in every partition of m words. */
static void permute_balanced(uint64_t *A, uint64_t n, uint64_t m, uint32_t d) {
    if (d > 8) {
        while (d > 8) {
            uint64_t k = (uint64_t)sqrt((double)m);
            for (uint64_t p = 0; p < n / m; ++p) equidistant_gather(&A[p * m], k, k);
            m = k;
            d /= 2;
        }
        basecase8(A, n);
    } else if (d == 8) {
        basecase8(A, n);
    } else if (d == 4) {
        basecase4(A, n);
    } else if (d == 2) {
        basecase2(A, n);
    }
}

/* permutevEB for perfect trees whose d is not a power of two:
 * gpu/src/mveb-cycles.cuh:233-297. */
static void permute_veb(uint64_t *A, uint64_t n, uint32_t d) {
    if (n == 1) return;
    uint32_t root_d, leaf_d;
    mveb_split(d, &root_d, &leaf_d);
    uint64_t r = ((uint64_t)1 << root_d) - 1;
    uint64_t l = ((uint64_t)1 << leaf_d) - 1;
    equidistant_gather(A, r, l);
    permute_balanced(&A[r], n - r, l, leaf_d);
    if (!is_pow2_levels(root_d))
        permute_veb(A, r, root_d);
    else
        permute_balanced(A, r, r, root_d);
}

static uint32_t bit_length(uint64_t x) {
    uint32_t d = 0;
    while (x) {
        ++d;
        x >>= 1;
    }
    return d;
}

/* permutevEB_nonperfect: gpu/src/mveb-cycles.cuh:302-414. */
static void permute_veb_nonperfect(uint64_t *A, uint64_t n, uint32_t d) {
    if (n == 1) return;
    uint32_t root_d, leaf_d;
    mveb_split(d, &root_d, &leaf_d);
    uint64_t r = ((uint64_t)1 << root_d) - 1;
    uint64_t l = ((uint64_t)1 << leaf_d) - 1;
    uint64_t num_full = (n - r) / l;
    uint64_t inc_n = n - r - num_full * l;

    equidistant_gather(A, num_full, l);
    if (num_full < r) shift_right(&A[num_full], n - num_full, r - num_full);

    if (root_d == leaf_d) {
        permute_balanced(A, n - inc_n, r, root_d);
    } else {
        permute_balanced(&A[r], num_full * l, l, leaf_d);
        if (!is_pow2_levels(root_d))
            permute_veb(A, r, root_d);
        else
            permute_balanced(A, r, r, root_d);
    }

    if (inc_n > 0) {
        /* inc_d = log2(inc_n) + 1 in double (:398); bit_length is the same value. */
        uint32_t inc_d = bit_length(inc_n);
        if (inc_n != ((uint64_t)1 << inc_d) - 1) {
            permute_veb_nonperfect(&A[n - inc_n], inc_n, inc_d);
        } else {
            if (!is_pow2_levels(inc_d))
                permute_veb(&A[n - inc_n], inc_n, inc_d);
            else
                permute_balanced(&A[n - inc_n], inc_n, inc_n, inc_d);
        }
    }
}

/* timePermutevEB: gpu/src/mveb-cycles.cuh:420-440.  d = log2((double)n) + 1 is
 * the bit length of n for every n below 2^52. */
int orc_permute_mveb(uint64_t *A, uint64_t n) {
    if (n == 0) return 0;
    uint32_t d = bit_length(n);
    if (n != ((uint64_t)1 << d) - 1) {
        permute_veb_nonperfect(A, n, d);
    } else {
        if (is_pow2_levels(d))
            permute_balanced(A, n, n, d);
        else
            permute_veb(A, n, d);
    }
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Standard van Emde Boas layout of the reference's CPU code                  */
/* ------------------------------------------------------------------------ */

/* cpu/src/veb-cycles.h:118-119: root_d = floor((d - 2)/2) + 1, leaf_d = the rest. */
static void veb_std_split(uint32_t d, uint32_t *root_d, uint32_t *leaf_d) {
    *root_d = (d - 2) / 2 + 1;
    *leaf_d = d - *root_d;
}

/* permutevEB: cpu/src/veb-cycles.h:33-57.  equidistant_gather_io (cpu/src/cycles.h:
 * 89-141) performs the cycles of equidistant_gather b at a time; the resulting
 * permutation is the same. */
static void permute_veb_std(uint64_t *A, uint64_t n, uint32_t d) {
    if (d <= 1) return;
    if (d % 2 == 0) {
        uint64_t m = ((uint64_t)1 << (d / 2)) - 1;
        equidistant_gather(A, m, m);
        for (uint64_t i = 0; i < n; i += m) permute_veb_std(&A[i], m, d / 2);
    } else {
        uint64_t r = ((uint64_t)1 << (d / 2)) - 1;
        uint64_t l = 2 * r + 1;
        equidistant_gather(A, r, l);
        permute_veb_std(A, r, d / 2);
        for (uint64_t i = r; i < n; i += l) permute_veb_std(&A[i], l, d / 2 + 1);
    }
}

/* permutevEB_nonperfect: cpu/src/veb-cycles.h:111-173 (2^(d-1) - 1 < n < 2^d - 1). */
static void permute_veb_std_nonperfect(uint64_t *A, uint64_t n, uint32_t d) {
    if (d <= 1) return;
    uint32_t root_d, leaf_d;
    veb_std_split(d, &root_d, &leaf_d);
    uint64_t r = ((uint64_t)1 << root_d) - 1;
    uint64_t l = ((uint64_t)1 << leaf_d) - 1;
    uint64_t num_full = (n - r) / l;
    uint64_t inc_n = n - r - num_full * l;
    equidistant_gather(A, num_full, l);
    if (num_full < r) shift_right(&A[num_full], n - num_full, r - num_full);
    uint64_t size;
    if (root_d == leaf_d) {
        size = (num_full + 1) * r;
        for (uint64_t i = 0; i < size; i += r) permute_veb_std(&A[i], r, root_d);
    } else {
        permute_veb_std(A, r, root_d);
        size = r + num_full * l;
        for (uint64_t i = r; i < size; i += l) permute_veb_std(&A[i], l, leaf_d);
    }
    if (inc_n > 0) {
        uint32_t inc_d = bit_length(inc_n);
        if (inc_n != ((uint64_t)1 << inc_d) - 1)
            permute_veb_std_nonperfect(&A[size], inc_n, inc_d);
        else
            permute_veb_std(&A[size], inc_n, inc_d);
    }
}

/* timePermutevEB: cpu/src/veb-cycles.h:380-395 (h = log2(n), d = h + 1 = the bit
 * length of n below 2^52). */
int orc_permute_veb_std(uint64_t *A, uint64_t n) {
    if (n == 0) return 0;
    uint32_t d = bit_length(n);
    if (n != ((uint64_t)1 << d) - 1)
        permute_veb_std_nonperfect(A, n, d);
    else
        permute_veb_std(A, n, d);
    return 0;
}

/* buildTable: cpu/src/query-veb.cpp:25-41 (standard split). */
void orc_build_table_std(orc_veb_table *table, uint64_t n, uint32_t d, uint32_t root_depth) {
    if (n == 1) return;
    uint32_t root_d, leaf_d;
    veb_std_split(d, &root_d, &leaf_d);
    uint64_t root_n = ((uint64_t)1 << root_d) - 1;
    uint64_t leaf_n = ((uint64_t)1 << leaf_d) - 1;
    uint32_t i = d - leaf_d;
    table[i].L = leaf_n;
    table[i].R = root_n;
    table[i].D = root_depth;
    orc_build_table_std(table, root_n, root_d, root_depth);
    orc_build_table_std(&table[i], leaf_n, leaf_d, i + root_depth);
}

/* Table-set sizing of cpu/test/query-veb-fixedN.cpp:37-84 (standard split). */
void orc_veb_tables_size_std(uint64_t n, uint32_t *num_tables, uint32_t *table_size) {
    uint32_t d = bit_length(n);
    uint32_t nt = 1, ts = d;
    if (n != ((uint64_t)1 << d) - 1) {
        uint64_t temp_n = n;
        uint32_t temp_d = d;
        while (temp_d >= 2) {
            uint32_t root_d, leaf_d;
            veb_std_split(temp_d, &root_d, &leaf_d);
            uint64_t r = ((uint64_t)1 << root_d) - 1;
            uint64_t l = ((uint64_t)1 << leaf_d) - 1;
            uint64_t num_full = (temp_n - r) / l;
            uint64_t inc_n = temp_n - r - num_full * l;
            if (inc_n == 0) break;
            uint32_t inc_d = bit_length(inc_n);
            ++nt;
            ts += inc_d;
            temp_n = inc_n;
            temp_d = inc_d;
            if (temp_n == ((uint64_t)1 << inc_d) - 1) break;
        }
    }
    *num_tables = nt;
    *table_size = ts;
}

/* Table-set construction of cpu/test/query-veb-fixedN.cpp:120-150, the tables
 * concatenated as the GPU driver lays them out (table_idx offsets). */
void orc_build_veb_tables_std(uint64_t n, orc_veb_table *tables, uint64_t *idx, uint32_t *table_idx) {
    uint32_t num_tables, table_size;
    orc_veb_tables_size_std(n, &num_tables, &table_size);
    memset(tables, 0, table_size * sizeof(orc_veb_table));
    uint32_t d = bit_length(n);
    orc_build_table_std(tables, n, d, 0);
    idx[num_tables - 1] = n;
    table_idx[0] = 0;
    uint64_t temp_n = n;
    uint32_t temp_d = d;
    for (uint32_t i = 1; i < num_tables; ++i) {
        table_idx[i] = table_idx[i - 1] + temp_d;
        uint32_t root_d, leaf_d;
        veb_std_split(temp_d, &root_d, &leaf_d);
        uint64_t r = ((uint64_t)1 << root_d) - 1;
        uint64_t l = ((uint64_t)1 << leaf_d) - 1;
        uint64_t num_full = (temp_n - r) / l;
        uint64_t inc_n = temp_n - r - num_full * l;
        uint32_t inc_d = bit_length(inc_n);
        orc_build_table_std(&tables[table_idx[i]], inc_n, inc_d, 0);
        idx[i - 1] = n - inc_n;
        temp_n = inc_n;
        temp_d = inc_d;
    }
}

/* ------------------------------------------------------------------------ */
/* Queries                                                                    */
/* ------------------------------------------------------------------------ */

/* searchBST: cpu/src/query-bst.h:29-41, gpu/src/query-bst.cuh:31-42. */
void orc_search_bst(const uint64_t *A, uint64_t n, const uint64_t *q, uint64_t nq, uint64_t *ans) {
    for (uint64_t k = 0; k < nq; ++k) {
        uint64_t query = q[k];
        uint64_t i = 0, res = n;
        while (i < n) {
            if (query == A[i]) {
                res = i;
                break;
            }
            i = 2 * i + 1 + (query > A[i]);
        }
        ans[k] = res;
    }
}

/* searchBtree: cpu/src/query-btree.h:33-54 (linear scan of each node).  The
 * reference scans b slots even in the last, partially filled node and reads past
 * n there; the scan below stops at n, which is what the reference computes when
 * the array is padded with keys larger than every query (the survey's pad). */
void orc_search_btree(const uint64_t *A, uint64_t n, uint64_t b, const uint64_t *q, uint64_t nq,
                      uint64_t *ans) {
    for (uint64_t k = 0; k < nq; ++k) {
        uint64_t query = q[k];
        uint64_t i = 0, j, res = n;
        int found = 0;
        while (i < n && !found) {
            for (j = 0; j < b; j++) {
                if (i + j >= n) break;
                uint64_t current = A[i + j];
                if (query == current) {
                    res = i + j;
                    found = 1;
                    break;
                } else if (query < current) {
                    break;
                }
            }
            if (found) break;
            i = (i + 1) * (b + 1) + j * b - 1;
        }
        ans[k] = res;
    }
}

/* buildTable: gpu/src/query-mveb.cu:25-47 (mvEB split). */
void orc_build_table(orc_veb_table *table, uint64_t n, uint32_t d, uint32_t root_depth) {
    if (n == 1) return;
    uint32_t root_d, leaf_d;
    mveb_split(d, &root_d, &leaf_d);
    uint64_t root_n = ((uint64_t)1 << root_d) - 1;
    uint64_t leaf_n = ((uint64_t)1 << leaf_d) - 1;
    uint32_t i = d - leaf_d;
    table[i].L = leaf_n;
    table[i].R = root_n;
    table[i].D = root_depth;
    orc_build_table(table, root_n, root_d, root_depth);
    orc_build_table(&table[i], leaf_n, leaf_d, i + root_depth);
}

/* Table-set sizing loop of gpu/test/query-mveb-fixedN.cu:45-97. */
void orc_veb_tables_size(uint64_t n, uint32_t *num_tables, uint32_t *table_size) {
    uint32_t d = bit_length(n);
    uint32_t nt = 1, ts = d;
    if (n != ((uint64_t)1 << d) - 1) {
        uint64_t temp_n = n;
        uint32_t temp_d = d;
        while (temp_d >= 2) {
            uint32_t root_d, leaf_d;
            mveb_split(temp_d, &root_d, &leaf_d);
            uint64_t r = ((uint64_t)1 << root_d) - 1;
            uint64_t l = ((uint64_t)1 << leaf_d) - 1;
            uint64_t num_full = (temp_n - r) / l;
            uint64_t inc_n = temp_n - r - num_full * l;
            if (inc_n == 0) break;
            uint32_t inc_d = bit_length(inc_n);
            ++nt;
            ts += inc_d;
            temp_n = inc_n;
            temp_d = inc_d;
            if (temp_n == ((uint64_t)1 << inc_d) - 1) break;
        }
    }
    *num_tables = nt;
    *table_size = ts;
}

/* Table-set construction of gpu/test/query-mveb-fixedN.cu:130-165. */
void orc_build_veb_tables(uint64_t n, orc_veb_table *tables, uint64_t *idx, uint32_t *table_idx) {
    uint32_t num_tables, table_size;
    orc_veb_tables_size(n, &num_tables, &table_size);
    memset(tables, 0, table_size * sizeof(orc_veb_table));
    uint32_t d = bit_length(n);
    orc_build_table(tables, n, d, 0);
    idx[num_tables - 1] = n;
    table_idx[0] = 0;
    uint64_t temp_n = n;
    uint32_t temp_d = d;
    for (uint32_t i = 1; i < num_tables; ++i) {
        table_idx[i] = table_idx[i - 1] + temp_d;
        uint32_t root_d, leaf_d;
        mveb_split(temp_d, &root_d, &leaf_d);
        uint64_t r = ((uint64_t)1 << root_d) - 1;
        uint64_t l = ((uint64_t)1 << leaf_d) - 1;
        uint64_t num_full = (temp_n - r) / l;
        uint64_t inc_n = temp_n - r - num_full * l;
        uint32_t inc_d = bit_length(inc_n);
        orc_build_table(&tables[table_idx[i]], inc_n, inc_d, 0);
        idx[i - 1] = n - inc_n;
        temp_n = inc_n;
        temp_d = inc_d;
    }
}

/* searchvEB: gpu/src/query-mveb.cuh:43-66 / cpu/src/query-veb.h:41-64.
 * The reference reads table[d] and writes pos[d] one past the end when a query
 * falls off a leaf (it only ever issues hits); here a descent that passes the
 * deepest level ends as "not found", which is the reference's documented result. */
static uint64_t search_veb_one(const uint64_t *A, const orc_veb_table *table, uint64_t n,
                               uint32_t d, uint64_t query, uint64_t offset, uint64_t limit,
                               int *fell_off) {
    uint64_t pos[65];
    uint32_t current_d = 0;
    uint64_t i = 1;
    uint64_t index = 0;
    pos[0] = 1;
    *fell_off = 0;
    while (index + offset < limit) {
        uint64_t current = A[offset + index];
        if (query == current) return offset + index;
        if (current_d + 1 >= d) {
            *fell_off = 1;
            return n;
        }
        i = 2 * i + (query > current);
        current_d++;
        pos[current_d] = pos[table[current_d].D] + table[current_d].R +
                         (i & table[current_d].R) * table[current_d].L;
        index = pos[current_d] - 1;
    }
    return n;
}

void orc_search_veb(const uint64_t *A, const orc_veb_table *table, uint64_t n, uint32_t d,
                    const uint64_t *q, uint64_t nq, uint64_t *ans) {
    for (uint64_t k = 0; k < nq; ++k) {
        int fell;
        ans[k] = search_veb_one(A, table, n, d, q[k], 0, n, &fell);
    }
}

/* searchvEB_nonperfect: gpu/src/query-mveb.cuh:173-213.  Table j describes the
 * perfect geometry of depth d_j; positions at or past idx[j] continue in the next
 * (incomplete) subtree. */
void orc_search_veb_nonperfect(const uint64_t *A, const orc_veb_table *tables, const uint64_t *idx,
                               const uint32_t *table_idx, uint64_t n, uint32_t d,
                               uint32_t num_tables, const uint64_t *q, uint64_t nq,
                               uint64_t *ans) {
    (void)d;
    for (uint64_t k = 0; k < nq; ++k) {
        uint64_t res = idx[num_tables - 1];
        uint64_t offset = 0;
        for (uint32_t j = 0; j < num_tables; ++j) {
            uint64_t sub_n = (j == 0 ? idx[num_tables - 1] : idx[num_tables - 1] - offset);
            uint32_t dj = bit_length(sub_n);
            int fell;
            uint64_t r = search_veb_one(A, &tables[table_idx[j]], n, dj, q[k], offset, idx[j], &fell);
            if (r != n) {
                res = r;
                break;
            }
            if (fell) break;
            offset = idx[j];
        }
        ans[k] = res;
    }
}

double orc_time_permute_btree(uint64_t *A, uint64_t n, uint64_t b) {
    struct timespec s, e;
    clock_gettime(CLOCK_MONOTONIC, &s);
    orc_permute_btree(A, n, b);
    clock_gettime(CLOCK_MONOTONIC, &e);
    return ((e.tv_sec * 1e9 + e.tv_nsec) - (s.tv_sec * 1e9 + s.tv_nsec)) / 1e6;
}
