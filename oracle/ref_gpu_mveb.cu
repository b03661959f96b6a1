// Thin extern "C" shim over the reference's own GPU mvEB code (TEST INFRASTRUCTURE).
// Compiled by oracle/Makefile for sm_100a against the reference sources where they
// lie; the built library (oracle/_ref/libref_gpu.so) is only used to pin the
// oracle's mvEB restatement on a B200 (tests/golden/make_mveb_golden.py).
#include "mveb-cycles.cuh"  // gpu/src/mveb-cycles.cuh: timePermutevEB (:420-440)
#include "query-mveb.cuh"   // gpu/src/query-mveb.cuh: vEB_table, buildTable

template <typename T>
static int permute_on_device(T *host, uint64_t n) {
    T *dev = nullptr;
    if (cudaMalloc(&dev, n * sizeof(T)) != cudaSuccess) return 1;
    cudaMemcpy(dev, host, n * sizeof(T), cudaMemcpyHostToDevice);
    timePermutevEB<T>(dev, n);
    cudaError_t e = cudaMemcpy(host, dev, n * sizeof(T), cudaMemcpyDeviceToHost);
    cudaFree(dev);
    return e == cudaSuccess ? 0 : 2;
}

extern "C" int ref_gpu_permute_mveb_u32(uint32_t *host, uint64_t n) { return permute_on_device(host, n); }
extern "C" int ref_gpu_permute_mveb_u64(uint64_t *host, uint64_t n) { return permute_on_device(host, n); }
// Host-only: gpu/src/query-mveb.cu:25-47.
extern "C" void ref_gpu_build_table(void *table, uint64_t n, uint32_t d, uint32_t root_depth) {
    buildTable(reinterpret_cast<vEB_table *>(table), n, d, root_depth);
}
