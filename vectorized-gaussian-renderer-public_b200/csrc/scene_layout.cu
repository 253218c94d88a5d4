// Spatial layout of a registered camera scene: a Morton order of the means
// and per-chunk bounds that let the projection skip, per camera, whole chunks
// of kProjectChunk Gaussians that lie outside its frustum.
//
// No counterpart in the reference, which projects every (camera, Gaussian)
// pair of a scene (renderer_cuda.cu:542-1091).  The layout changes no
// output: a permuted scene reports every Gaussian by its original id
// (vgr_scene.gaussian_ids), which is what the tile sort breaks depth ties
// with and what indexes the semantic table, and a chunk is skipped only when
// the projection's own conservative early cull would reject every Gaussian
// in it (the bound is derived from that cull below).
#include <cuda_runtime.h>

#include <climits>
#include <cstddef>

#include "../../include/vgr_b200.h"
#include "vgr_api_internal.h"
#include "vgr_kernels.h"

namespace vgr {
namespace {

struct OrderHeader {
  uint32_t bounds_bits[6];   // order-preserving codes of the means' AABB
  uint32_t pad[2];
  int64_t sort_counters[5];  // [1] = items to sort (raw-key onesweep)
};

struct OrderLayout {
  int64_t header;
  int64_t keys_a;
  int64_t keys_b;
  int64_t vals_a;
  int64_t vals_b;
  int64_t sort;
  ScratchLayout sort_layout;
  int64_t total;
};

OrderLayout make_order_layout(int64_t count) {
  OrderLayout l{};
  int64_t off = 0;
  auto take = [&](int64_t bytes) {
    const int64_t at = off;
    off = align_up(off + bytes, 256);
    return at;
  };
  l.header = take(sizeof(OrderHeader));
  l.keys_a = take(count * 8);
  l.keys_b = take(count * 8);
  l.vals_a = take(count * 4);
  l.vals_b = take(count * 4);
  l.sort_layout = make_scratch_layout(count > 0 ? count : 1, 0, true);
  l.sort = take(l.sort_layout.total);
  l.total = off;
  return l;
}

__global__ void order_init_kernel(unsigned char* base, OrderLayout l, int64_t count) {
  OrderHeader* h = reinterpret_cast<OrderHeader*>(base + l.header);
  for (int a = 0; a < 3; ++a) {
    h->bounds_bits[a] = 0xffffffffu;
    h->bounds_bits[3 + a] = 0u;
  }
  for (int k = 0; k < 5; ++k) h->sort_counters[k] = 0;
  h->sort_counters[1] = count;
  uint32_t* words = reinterpret_cast<uint32_t*>(base + l.sort + l.sort_layout.header);
  for (int k = 0; k < 32; ++k) words[k] = 0u;
  uint32_t* hist = reinterpret_cast<uint32_t*>(base + l.sort + l.sort_layout.sort_hist);
  for (int k = 0; k < kMaxSortPasses * kRadixBins; ++k) hist[k] = 0u;
}

__global__ void __launch_bounds__(256) order_bounds_kernel(const float* __restrict__ means,
                                                           int64_t count, OrderHeader* h) {
  uint32_t lo[3] = {0xffffffffu, 0xffffffffu, 0xffffffffu};
  uint32_t hi[3] = {0u, 0u, 0u};
  for (int64_t g = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; g < count;
       g += static_cast<int64_t>(gridDim.x) * blockDim.x) {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const uint32_t v = float_order(means[g * 3 + a]);
      lo[a] = min(lo[a], v);
      hi[a] = max(hi[a], v);
    }
  }
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    lo[a] = __reduce_min_sync(0xffffffffu, lo[a]);
    hi[a] = __reduce_max_sync(0xffffffffu, hi[a]);
    if ((threadIdx.x & 31) == 0) {
      atomicMin(&h->bounds_bits[a], lo[a]);
      atomicMax(&h->bounds_bits[3 + a], hi[a]);
    }
  }
}

// 30-bit Morton key of each mean over the AABB; value = index.
__global__ void __launch_bounds__(256) order_keys_kernel(const float* __restrict__ means,
                                                         int64_t count, const OrderHeader* h,
                                                         uint64_t* keys, int32_t* vals) {
  const int64_t g = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (g >= count) return;
  uint32_t q[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const float low = order_float(h->bounds_bits[a]);
    const float extent = fmaxf(order_float(h->bounds_bits[3 + a]) - low, 1.0e-12f);
    const float normalized = fminf(fmaxf((means[g * 3 + a] - low) / extent, 0.0f), 1.0f);
    q[a] = static_cast<uint32_t>(normalized * 1023.0f + 0.5f);
  }
  keys[g] = expand_bits(q[0]) | (expand_bits(q[1]) << 1) | (expand_bits(q[2]) << 2);
  vals[g] = static_cast<int32_t>(g);
}

// Position of (x, y), both below 2^15, along the 2D Hilbert curve of order
// 15 (30 bits): the quadrant index of each level from the top, each level's
// quadrant reflected and transposed so consecutive positions stay adjacent
// (Hilbert's construction, as in Skilling's and the classic xy-to-d forms).
__device__ __forceinline__ uint64_t hilbert_index(uint32_t x, uint32_t y) {
  constexpr uint32_t kSide = 1u << 15;
  uint64_t d = 0;
  for (uint32_t s = kSide >> 1; s > 0; s >>= 1) {
    const uint32_t rx = (x & s) ? 1u : 0u;
    const uint32_t ry = (y & s) ? 1u : 0u;
    d += static_cast<uint64_t>(s) * s * ((3u * rx) ^ ry);
    if (ry == 0) {
      if (rx == 1) {
        x = kSide - 1 - x;
        y = kSide - 1 - y;
      }
      const uint32_t t = x;
      x = y;
      y = t;
    }
  }
  return d;
}

// 30-bit Hilbert key of each direction's (azimuth, elevation) on one angular
// grid of 2 pi / 32768 per step on both axes (isotropic in angle, so 32
// consecutive keys form a compact patch of directions: on a spinning LiDAR's
// 2048 x 128 grid a median of 8 azimuths x 4 beams, against 13 x 4 with a
// Morton key, whose jumps between quadrants split some patches); value =
// index.  A non-finite direction gets key 0.
__global__ void __launch_bounds__(256) order_angle_keys_kernel(const float* __restrict__ dirs,
                                                               int64_t count, uint64_t* keys,
                                                               int32_t* vals) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const float x = dirs[i * 3 + 0], y = dirs[i * 3 + 1], z = dirs[i * 3 + 2];
  const float norm = sqrtf(x * x + y * y + z * z);
  uint64_t key = 0;
  if (isfinite(norm) && norm > 0.0f) {
    constexpr float kPi = 3.14159265358979f;
    constexpr float kStep = 32768.0f / (2.0f * kPi);
    const float az = atan2f(y, x);                                // [-pi, pi]
    const float el = asinf(fminf(fmaxf(z / norm, -1.0f), 1.0f));  // [-pi/2, pi/2]
    const uint32_t qa = min(static_cast<uint32_t>(fmaxf((az + kPi) * kStep, 0.0f)), 32767u);
    const uint32_t qe = min(static_cast<uint32_t>(fmaxf((el + 0.5f * kPi) * kStep, 0.0f)), 32767u);
    key = hilbert_index(qa, qe);
  }
  keys[i] = key;
  vals[i] = static_cast<int32_t>(i);
}

__global__ void __launch_bounds__(256) order_copy_kernel(const int32_t* __restrict__ sorted,
                                                         int64_t count, int32_t* order) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < count) order[i] = sorted[i];
}

// One CTA per chunk: AABB of the means and the largest covariance trace.
constexpr int kBoundsThreads = 128;
__global__ void __launch_bounds__(kBoundsThreads) chunk_bounds_kernel(
    const float* __restrict__ means, const float* __restrict__ covariances, int64_t count,
    float4* __restrict__ bounds) {
  __shared__ float s_red[7][kBoundsThreads / 32];
  const int64_t begin = static_cast<int64_t>(blockIdx.x) * kProjectChunk;
  float lo[3] = {__int_as_float(0x7f800000), __int_as_float(0x7f800000), __int_as_float(0x7f800000)};
  float hi[3] = {-__int_as_float(0x7f800000), -__int_as_float(0x7f800000), -__int_as_float(0x7f800000)};
  float trace = 0.0f;
  for (int i = threadIdx.x; i < kProjectChunk; i += kBoundsThreads) {
    const int64_t g = begin + i;
    if (g >= count) break;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const float m = means[g * 3 + a];
      lo[a] = fminf(lo[a], m);
      hi[a] = fmaxf(hi[a], m);
    }
    const float* s = covariances + g * 6;
    trace = fmaxf(trace, s[0] + s[3] + s[5]);
  }
  float v[7] = {lo[0], lo[1], lo[2], -hi[0], -hi[1], -hi[2], -trace};
#pragma unroll
  for (int k = 0; k < 7; ++k) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[k] = fminf(v[k], __shfl_xor_sync(0xffffffffu, v[k], o));
    if ((threadIdx.x & 31) == 0) s_red[k][threadIdx.x >> 5] = v[k];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < 7; ++k) {
      for (int w = 1; w < kBoundsThreads / 32; ++w) s_red[k][0] = fminf(s_red[k][0], s_red[k][w]);
    }
    // A non-finite mean or trace disables culling for the chunk.
    bounds[blockIdx.x * 2 + 0] = make_float4(s_red[0][0], s_red[1][0], s_red[2][0], -s_red[6][0]);
    bounds[blockIdx.x * 2 + 1] = make_float4(-s_red[3][0], -s_red[4][0], -s_red[5][0], 0.0f);
  }
}

// One warp per cluster of kProjectCluster Gaussians (lane = Gaussian): the
// same bounds as chunk_bounds_kernel; a cluster past the end of the scene
// gets an empty box (lo = +inf, hi = -inf) and trace 0.
__global__ void __launch_bounds__(256) cluster_bounds_kernel(const float* __restrict__ means,
                                                             const float* __restrict__ covariances,
                                                             int64_t count, int64_t clusters,
                                                             float4* __restrict__ bounds) {
  const int64_t cluster = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  if (cluster >= clusters) return;  // warp-uniform
  const int lane = threadIdx.x & 31;
  const int64_t g = cluster * kProjectCluster + lane;
  const float inf = __int_as_float(0x7f800000);
  float v[7] = {inf, inf, inf, inf, inf, inf, 0.0f};  // lo xyz, -hi xyz, -trace
  if (g < count) {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      v[a] = means[g * 3 + a];
      v[3 + a] = -v[a];
    }
    const float* s = covariances + g * 6;
    v[6] = -(s[0] + s[3] + s[5]);
  }
#pragma unroll
  for (int k = 0; k < 7; ++k) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[k] = fminf(v[k], __shfl_xor_sync(0xffffffffu, v[k], o));
  }
  if (lane == 0) {
    // A non-finite mean or trace disables culling for the cluster.
    bounds[cluster * 2 + 0] = make_float4(v[0], v[1], v[2], -v[6]);
    bounds[cluster * 2 + 1] = make_float4(-v[3], -v[4], -v[5], 0.0f);
  }
}

unsigned grid_for(int64_t items, int threads) {
  const int64_t blocks = (items + threads - 1) / threads;
  return static_cast<unsigned>(blocks < 1 ? 1 : blocks);
}

}  // namespace
}  // namespace vgr

using namespace vgr;

extern "C" int64_t vgr_scene_spatial_order_temp_bytes(int64_t gaussian_count) {
  if (gaussian_count <= 0 || gaussian_count > INT_MAX) {
    return fail(VGR_ERR_INVALID_ARGUMENT, "a scene needs 1..INT_MAX Gaussians");
  }
  return make_order_layout(gaussian_count).total;
}

namespace {

// Stable order of `count` points by a 30-bit key: the Morton key of the 3D
// points over their bounding box, or (angular) the Hilbert key of the
// directions' azimuth and elevation.
int morton_order(const float* means, int64_t count, int32_t* order, void* temp, int64_t temp_bytes,
                 void* stream_ptr, bool angular) {
  if (!means || !order || !temp) return fail(VGR_ERR_INVALID_ARGUMENT, "arguments must be non-null");
  if (count <= 0 || count > INT_MAX) return fail(VGR_ERR_INVALID_ARGUMENT, "an order needs 1..INT_MAX items");
  if ((reinterpret_cast<uintptr_t>(temp) & 255) != 0) {
    return fail(VGR_ERR_INVALID_ARGUMENT, "temp buffer must be 256-byte aligned");
  }
  const OrderLayout layout = make_order_layout(count);
  if (temp_bytes < layout.total) {
    return fail(VGR_ERR_SCRATCH_TOO_SMALL, "spatial order temp holds %lld bytes, needs %lld",
                static_cast<long long>(temp_bytes), static_cast<long long>(layout.total));
  }
  int sms = 0;
  int rc = device_sms(&sms);
  if (rc != VGR_OK) return rc;
  cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
  unsigned char* base = static_cast<unsigned char*>(temp);
  OrderHeader* h = reinterpret_cast<OrderHeader*>(base + layout.header);
  order_init_kernel<<<1, 1, 0, stream>>>(base, layout, count);
  if ((rc = check_launch("spatial order: init")) != VGR_OK) return rc;
  unsigned bgrid = grid_for(count, 256);
  if (bgrid > static_cast<unsigned>(sms * 4)) bgrid = static_cast<unsigned>(sms * 4);
  if (!angular) {
    order_bounds_kernel<<<bgrid, 256, 0, stream>>>(means, count, h);
    if ((rc = check_launch("spatial order: bounds")) != VGR_OK) return rc;
  }
  uint64_t* kin = reinterpret_cast<uint64_t*>(base + layout.keys_a);
  uint64_t* kout = reinterpret_cast<uint64_t*>(base + layout.keys_b);
  int32_t* vin = reinterpret_cast<int32_t*>(base + layout.vals_a);
  int32_t* vout = reinterpret_cast<int32_t*>(base + layout.vals_b);
  if (angular) {
    order_angle_keys_kernel<<<grid_for(count, 256), 256, 0, stream>>>(means, count, kin, vin);
  } else {
    order_keys_kernel<<<grid_for(count, 256), 256, 0, stream>>>(means, count, h, kin, vin);
  }
  if ((rc = check_launch("spatial order: keys")) != VGR_OK) return rc;

  // Stable raw-key radix sort of the 30-bit keys (the onesweep of the LBVH).
  SortParams so{};
  so.scratch = base + layout.sort;
  so.layout = layout.sort_layout;
  so.counters = reinterpret_cast<const int64_t*>(base + layout.header + offsetof(OrderHeader, sort_counters));
  so.capacity = count;
  so.map.raw = 1;
  so.map.total_bits = 30;
  so.passes = 4;
  so.keys_in = kin;
  const int64_t parts = layout.sort_layout.max_partitions;
  sort_histogram_kernel<<<static_cast<unsigned>(parts < sms * 4 ? parts : sms * 4), kSortThreads, 0,
                          stream>>>(so);
  if ((rc = check_launch("spatial order: sort histogram")) != VGR_OK) return rc;
  int sort_ctas = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&sort_ctas, sort_onesweep_kernel, kSortThreads,
                                                kSortDynamicSmem);
  if (sort_ctas < 1) sort_ctas = 1;
  int64_t sgrid = static_cast<int64_t>(sms) * sort_ctas;
  if (sgrid > parts) sgrid = parts;
  for (int pass = 0; pass < so.passes; ++pass) {
    so.pass = pass;
    so.keys_in = kin;
    so.values_in = vin;
    so.keys_out = kout;
    so.values_out = vout;
    sort_onesweep_kernel<<<static_cast<unsigned>(sgrid), kSortThreads, kSortDynamicSmem, stream>>>(so);
    if ((rc = check_launch("spatial order: sort pass")) != VGR_OK) return rc;
    uint64_t* tk = kin; kin = kout; kout = tk;
    int32_t* tv = vin; vin = vout; vout = tv;
  }
  order_copy_kernel<<<grid_for(count, 256), 256, 0, stream>>>(vin, count, order);
  return check_launch("spatial order: copy");
}

}  // namespace

extern "C" int vgr_scene_spatial_order(const float* means, int64_t count, int32_t* order,
                                       void* temp, int64_t temp_bytes, void* stream_ptr) {
  return morton_order(means, count, order, temp, temp_bytes, stream_ptr, false);
}

extern "C" int64_t vgr_lidar_ray_order_temp_bytes(int64_t rays) {
  if (rays <= 0 || rays > INT_MAX) return fail(VGR_ERR_INVALID_ARGUMENT, "an order needs 1..INT_MAX rays");
  return make_order_layout(rays).total;
}

extern "C" int vgr_lidar_ray_order(const float* ray_directions, int64_t rays, int32_t* order, void* temp,
                                   int64_t temp_bytes, void* stream_ptr) {
  return morton_order(ray_directions, rays, order, temp, temp_bytes, stream_ptr, true);
}

extern "C" int vgr_scene_chunk_bounds(const float* means, const float* covariances, int64_t count,
                                      float* bounds, void* stream_ptr) {
  if (!means || !covariances || !bounds) return fail(VGR_ERR_INVALID_ARGUMENT, "arguments must be non-null");
  if (count <= 0 || count > INT_MAX) return fail(VGR_ERR_INVALID_ARGUMENT, "a scene needs 1..INT_MAX Gaussians");
  if ((reinterpret_cast<uintptr_t>(bounds) & 15) != 0) {
    return fail(VGR_ERR_INVALID_ARGUMENT, "bounds must be 16-byte aligned");
  }
  const int64_t chunks = (count + kProjectChunk - 1) / kProjectChunk;
  chunk_bounds_kernel<<<static_cast<unsigned>(chunks), kBoundsThreads, 0,
                        static_cast<cudaStream_t>(stream_ptr)>>>(means, covariances, count,
                                                                 reinterpret_cast<float4*>(bounds));
  return check_launch("chunk bounds");
}

extern "C" int vgr_scene_cluster_bounds(const float* means, const float* covariances, int64_t count,
                                        float* bounds, void* stream_ptr) {
  if (!means || !covariances || !bounds) return fail(VGR_ERR_INVALID_ARGUMENT, "arguments must be non-null");
  if (count <= 0 || count > INT_MAX) return fail(VGR_ERR_INVALID_ARGUMENT, "a scene needs 1..INT_MAX Gaussians");
  if ((reinterpret_cast<uintptr_t>(bounds) & 15) != 0) {
    return fail(VGR_ERR_INVALID_ARGUMENT, "bounds must be 16-byte aligned");
  }
  const int64_t clusters = (count + kProjectChunk - 1) / kProjectChunk * kProjectClusters;
  cluster_bounds_kernel<<<grid_for(clusters * 32, 256), 256, 0, static_cast<cudaStream_t>(stream_ptr)>>>(
      means, covariances, count, clusters, reinterpret_cast<float4*>(bounds));
  return check_launch("cluster bounds");
}
