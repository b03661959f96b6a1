// Internal declarations of the batched mode (batched.cu).
#pragma once

#include "internal.h"

namespace tl {
int batch_plan_create(const int64_t *dev_offsets, uint32_t num, uint64_t b, uint32_t key_bytes, cudaStream_t st,
                      tl_batch_plan **out);
int batch_plan_destroy(tl_batch_plan *plan);
int batch_workspace_bytes(const tl_batch_plan *plan, uint64_t *bytes);
int batch_permute(const tl_batch_plan *plan, void *dev_keys, void *dev_ws, uint64_t ws_bytes, cudaStream_t st);
int batch_status(const tl_batch_plan *plan, const void *dev_ws, cudaStream_t st);
int batch_ordered(const tl_batch_plan *plan, uint64_t *instances, uint64_t *keys);
int batch_query_workspace_bytes(const tl_batch_plan *plan, uint64_t q, uint64_t *bytes);
int batch_query(const tl_batch_plan *plan, const void *dev_keys, const void *dev_queries, const uint32_t *dev_inst,
                uint64_t q, uint64_t *dev_answers, void *dev_ws, uint64_t ws_bytes, cudaStream_t st, float *ms);
int batch_set_tuning(tl_batch_plan *plan, const uint32_t *tile_keys, const uint32_t *pin_levels, uint32_t query_chunk,
                     uint32_t threads, const int64_t *dev_offsets, cudaStream_t st);
int batch_get_tuning(const tl_batch_plan *plan, uint32_t *tile_keys, uint32_t *pin_levels, uint32_t *query_chunk,
                     uint32_t *threads);
int batch_autotune(tl_batch_plan *plan, const int64_t *dev_offsets, void *dev_keys, const void *dev_queries,
                   const uint32_t *dev_inst, uint64_t q, cudaStream_t st, char *report, size_t report_len);
}  // namespace tl
