// A host program written against the reference's GPU API (the template
// functions of algoparc/Tree-Layouts gpu/src, as its drivers in gpu/test call
// them: build-*.cu, query-*-fixedN.cu), compiled against tree_layouts.cuh and
// linked with -ltreelayouts instead of the reference's headers.  Used by
// tests/test_dropin_header.py.
//
//   dropin_driver OUT_DIR
//
// For each case: n sorted keys 1..n (as the reference's initSortedList fills
// them) are copied to the device, permuted with timePermuteBST / Btree / vEB,
// copied back and written to OUT_DIR/<layout>_<n>_<b>_<bits>.bin (raw, little
// endian); then the matching timeQuery* runs 100000 generated queries over the
// same keys.  Prints one line per case: name, permute ms, query ms.  Exits
// non-zero on any negative (failed) time.
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "tree_layouts.cuh"

template <typename TYPE>
static void init_sorted(TYPE *A, uint64_t n) {
    for (uint64_t i = 0; i < n; ++i) A[i] = (TYPE)(i + 1);
}

template <typename TYPE>
static bool write_file(const std::string &path, const TYPE *A, uint64_t n) {
    FILE *f = fopen(path.c_str(), "wb");
    if (!f) return false;
    const bool ok = fwrite(A, sizeof(TYPE), n, f) == n;
    return fclose(f) == 0 && ok;
}

// vEB tables as the reference's query driver holds them: one table for a
// perfect tree (buildTable), else one per division with idx / table_idx.
struct DeviceTables {
    vEB_table *tables = nullptr;
    uint64_t *idx = nullptr;
    uint32_t *table_idx = nullptr;
    uint32_t num_tables = 0, d = 0;
};

static bool make_tables(uint64_t n, DeviceTables &t) {
    uint32_t nt = 0, total = 0, d = 0;
    if (tl_veb_tables_size(n, &nt, &total, &d) != TL_SUCCESS) return false;
    std::vector<vEB_table> tab(total);
    std::vector<uint64_t> idx(nt);
    std::vector<uint32_t> tidx(nt);
    if (nt == 1) {
        buildTable(tab.data(), n, d, 0);
    } else if (tl_build_veb_tables(n, tab.data(), idx.data(), tidx.data()) != TL_SUCCESS) {
        return false;
    }
    t.num_tables = nt;
    t.d = d;
    cudaMalloc(&t.tables, total * sizeof(vEB_table));
    cudaMalloc(&t.idx, nt * sizeof(uint64_t));
    cudaMalloc(&t.table_idx, nt * sizeof(uint32_t));
    cudaMemcpy(t.tables, tab.data(), total * sizeof(vEB_table), cudaMemcpyHostToDevice);
    cudaMemcpy(t.idx, idx.data(), nt * sizeof(uint64_t), cudaMemcpyHostToDevice);
    cudaMemcpy(t.table_idx, tidx.data(), nt * sizeof(uint32_t), cudaMemcpyHostToDevice);
    return true;
}

template <typename TYPE>
static int run_case(const std::string &out, const char *layout, uint64_t n, uint64_t b) {
    const uint64_t q = 100000;
    TYPE *A = (TYPE *)malloc(n * sizeof(TYPE));
    TYPE *dev_A;
    cudaMalloc(&dev_A, n * sizeof(TYPE));
    init_sorted<TYPE>(A, n);
    cudaMemcpy(dev_A, A, n * sizeof(TYPE), cudaMemcpyHostToDevice);
    const std::string lay(layout);
    double pms = -1.0;
    if (lay == "bst") pms = timePermuteBST<TYPE>(dev_A, n);
    if (lay == "btree") pms = timePermuteBtree<TYPE>(dev_A, n, b);
    if (lay == "mveb") pms = timePermutevEB<TYPE>(dev_A, n);
    cudaMemcpy(A, dev_A, n * sizeof(TYPE), cudaMemcpyDeviceToHost);
    const std::string path = out + "/" + lay + "_" + std::to_string(n) + "_" + std::to_string(b) + "_" +
                             std::to_string(8 * sizeof(TYPE)) + ".bin";
    if (!write_file(path, A, n)) pms = -1.0;
    // the query functions take the host copy of the layout and copy it over
    // dev_A first, as the reference's do (its query drivers permute, copy the
    // layout back into A, then call timeQuery*)
    float qms = -1.f;
    if (lay == "bst") {
        qms = timeQueryBST<TYPE>(A, dev_A, n, q);
    } else if (lay == "btree") {
        qms = timeQueryBtree<TYPE>(A, dev_A, n, b, q);
    } else {
        DeviceTables t;
        if (make_tables(n, t)) {
            if (t.num_tables == 1)
                qms = timeQueryvEB<TYPE>(A, dev_A, t.tables, n, t.d, q);
            else
                qms = timeQueryvEB_nonperfect<TYPE>(A, dev_A, t.tables, t.idx, t.table_idx, n, t.d, t.num_tables,
                                                    q);
        }
        cudaFree(t.tables);
        cudaFree(t.idx);
        cudaFree(t.table_idx);
    }
    init_sorted<TYPE>(A, n);
    const float sms = timeQuery<TYPE>(A, dev_A, n, q);  // binary search over the sorted keys
    printf("%s n=%llu b=%llu bits=%d permute_ms=%.3f query_ms=%.3f search_ms=%.3f\n", layout,
           (unsigned long long)n, (unsigned long long)b, (int)(8 * sizeof(TYPE)), pms, qms, sms);
    free(A);
    cudaFree(dev_A);
    return (pms < 0 || qms < 0 || sms < 0) ? 1 : 0;
}

int main(int argc, char *argv[]) {
    if (argc != 2) {
        fprintf(stderr, "Usage: %s <output directory>\n", argv[0]);
        return 2;
    }
    const std::string out(argv[1]);
    int bad = 0;
    bad += run_case<uint32_t>(out, "btree", 1000003, 16);
    bad += run_case<uint64_t>(out, "btree", 70001, 8);
    bad += run_case<uint32_t>(out, "bst", (1u << 20) - 1, 1);
    bad += run_case<uint64_t>(out, "bst", 777777, 1);
    bad += run_case<uint32_t>(out, "mveb", (1u << 20) - 1, 0);
    bad += run_case<uint32_t>(out, "mveb", 3000017, 0);
    bad += run_case<uint64_t>(out, "mveb", 100003, 0);
    return bad ? 1 : 0;
}
