// Internal declarations of the learned-start module (learned.cu).
#pragma once

#include "internal.h"

namespace tl {
int rank_model_train(const uint64_t *keys, uint64_t n, const tl_rank_train_config *cfg, tl_rank_model *out,
                     tl_rank_leaf *leaves, cudaStream_t st);
int rank_model_root_eval(const tl_rank_model *m, const float *x, uint32_t count, float *out, uint32_t *pieces);
int rank_model_predict(const tl_rank_model *m, const tl_rank_leaf *leaves, const uint64_t *keys, uint64_t q,
                       uint64_t *rank, uint32_t *eps, cudaStream_t st);
int rank_model_gradient(const tl_rank_model *m, const float *dx, const float *dy, uint32_t count, float *grad,
                        float *loss, cudaStream_t st);
int query_btree_learned(const uint64_t *A, uint64_t n, uint64_t b, const tl_rank_model *m,
                        const tl_rank_leaf *leaves, const uint64_t *Q, uint64_t q, uint64_t *ans,
                        unsigned long long *stats, cudaStream_t st, float *ms);
}  // namespace tl
