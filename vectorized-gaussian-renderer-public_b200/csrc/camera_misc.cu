// Scene covariance precompute and logical-batch chunk bookkeeping.
#include "vgr_camera.cuh"
#include "vgr_misc.h"

namespace vgr {

// Object-space covariance Sigma = R diag(s^2) R^T from a WXYZ quaternion and
// activated scales (renderer_cuda.cu:112-143,492-540).  The quaternion is
// normalised by 1/sqrt(max(|q|^2, 1e-20)) with IEEE division and square root.
__global__ void __launch_bounds__(256) precompute_covariances_kernel(
    const float* __restrict__ scales, const float* __restrict__ rotations, int64_t count,
    float* __restrict__ covariances) {
  const int64_t g = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (g >= count) return;
  float cov[6];
  covariance_from_quaternion(rotations[g * 4 + 0], rotations[g * 4 + 1], rotations[g * 4 + 2],
                             rotations[g * 4 + 3], scales[g * 3 + 0], scales[g * 3 + 1],
                             scales[g * 3 + 2], cov);
#pragma unroll
  for (int k = 0; k < 6; ++k) covariances[g * 6 + k] = cov[k];
}

// Logical -> physical chunk bookkeeping (renderer_cuda.cu:2307-2360).
__global__ void mark_active_kernel(const int64_t* __restrict__ ids, int64_t count,
                                   int32_t* __restrict__ mask, int64_t logical_batch) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const int64_t cam = ids[i];
  if (cam >= 0 && cam < logical_batch) atomicExch(mask + cam, 1);
}

__global__ void build_chunk_ids_kernel(const int32_t* __restrict__ mask, int64_t logical_batch,
                                       int64_t physical_batch, int64_t slot_count,
                                       int64_t columns, int64_t* __restrict__ chunk_ids) {
  const int64_t slot = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (slot >= slot_count) return;
  const int64_t row = slot / physical_batch;
  const int64_t col = slot - row * physical_batch;
  chunk_ids[row * columns + col] =
      (slot < logical_batch && mask[slot] != 0) ? (slot % physical_batch) : -1;
}

__global__ void aggregate_counters_kernel(const int64_t* __restrict__ chunk_counters,
                                          int64_t stride, int64_t chunks,
                                          int64_t* __restrict__ counters,
                                          int64_t* __restrict__ physical) {
  const int c = threadIdx.x;
  if (c >= 5) return;
  int64_t total = 0, maximum = 0;
  for (int64_t k = 0; k < chunks; ++k) {
    const int64_t v = chunk_counters[k * stride + c];
    total += v;
    maximum = v > maximum ? v : maximum;
  }
  counters[c] = total;
  physical[c] = maximum;
}

}  // namespace vgr
