// Reverse permutations (layout -> sorted order) and the geometry they share
// with the forward permutation (permute.cu, unpermute.cu).
#pragma once

#include "btree_plan.cuh"
#include "mveb_plan.cuh"

namespace tl {

// The tile geometry of a permutation of (layout, n, b, key_bytes), with the
// B-tree's fixed right-to-left schedule (btree_stream_regime's regimes and
// btree_group_run's runs then cover every key) or the vEB plan.
struct PermuteGeometry {
    int layout = 0;
    uint32_t key_bytes = 8;
    uint64_t n = 0, tile_keys = 0, ntiles = 0;
    BtreeStream bs;
    MvebParams mp;
};

int permute_geometry(int layout, uint64_t n, uint64_t b, uint32_t key_bytes, PermuteGeometry &geo);

int unpermute(int layout, void *dev_A, uint64_t n, uint64_t b, uint32_t key_bytes, void *dev_ws, uint64_t ws_bytes,
              cudaStream_t st, float *ms);
int unpermute_workspace_bytes(int layout, uint64_t n, uint64_t b, uint32_t key_bytes, uint64_t *bytes);
int emulate_unpermute(int layout, uint64_t n, uint64_t b, uint64_t *A);

}  // namespace tl
