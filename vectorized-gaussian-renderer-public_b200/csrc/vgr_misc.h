// Declarations of the small utility kernels.
#pragma once

#include <stdint.h>

namespace vgr {

__global__ void precompute_covariances_kernel(const float* scales, const float* rotations,
                                              int64_t count, float* covariances);
__global__ void mark_active_kernel(const int64_t* ids, int64_t count, int32_t* mask,
                                   int64_t logical_batch);
__global__ void build_chunk_ids_kernel(const int32_t* mask, int64_t logical_batch,
                                       int64_t physical_batch, int64_t slot_count,
                                       int64_t columns, int64_t* chunk_ids);
__global__ void aggregate_counters_kernel(const int64_t* chunk_counters, int64_t stride,
                                          int64_t chunks, int64_t* counters, int64_t* physical);

}  // namespace vgr
