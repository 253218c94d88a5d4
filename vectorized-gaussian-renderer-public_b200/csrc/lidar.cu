// Gaussian-surfel LiDAR: LBVH build and batched first-return tracing.
//
// Equation of the reference LiDAR
// (src/isaacsim_gaussian_renderer/native/lidar_renderer_cuda.cu):
//  * candidate test (:329-421): normal = axis of the smallest scale, reject
//    when smallest / min(tangent scales) > planarity or the smallest scale is
//    not positive, |cos| >= min incidence, plane distance t in [near, far],
//    tangent Mahalanobis q <= sigma^2, weight = opacity * exp(-q/2) *
//    confidence >= threshold, intensity = clamp(reflectivity * exp(-q/2) *
//    |cos|);
//  * per return (:423-635,795-836): nearest candidate with t beyond the
//    previous cluster end, then a cluster window [t, t + max(abs, rel t)]
//    reduced in double precision (weighted range and intensity; semantic =
//    largest summed weight, ties -> smallest id; more distinct labels than
//    slots -> semantic overflow, no return);
//  * no-hit contract and call/error counters (:637-851).
//
// B200 structure.  Build: Gaussians that can never pass the planarity test
// are keyed past every Morton code, so one stable radix sort (the camera
// path's onesweep, raw-key mode) both orders the planar surfels along the
// 30-bit Morton curve (reference quantisation, :171-193) and moves the rest
// out of the way; the planar surfels are gathered into 80-byte records in
// that order, packed into leaves of 8 or 16, and a Karras radix tree is
// built over the leaves (64-bit leaf keys = Morton code << 32 | leaf index)
// with one CTA-free bottom-up refit whose second-arriving child computes the
// union.  Nodes store both child boxes, so one 64-byte load tests both
// children.  Trace: one thread per (active sensor, ray), near-first stack
// traversal for the nearest candidate and a window traversal for the
// cluster, as in the reference.
#include <cuda_runtime.h>
#include <math_constants.h>

#include <climits>
#include <cmath>

#include "../../include/vgr_b200.h"
#include "vgr_api_internal.h"
#include "vgr_kernels.h"

namespace vgr {
namespace {

constexpr int kLidarThreads = 256;
constexpr int kTraceThreads = 64;
constexpr int kMaxStack = 64;
constexpr int kMaxSemanticSlots = 32;
constexpr int kMaxCluster = 16;  // candidates kept per cluster window in one traversal
constexpr uint32_t kNonPlanarKey = 1u << 30;

struct __align__(16) Surfel {
  float4 m;   // mean xyz, max(scale0, scale1)^2 (all the distance pre-test reads)
  float4 n;   // normal xyz, surface confidence
  float4 a0;  // tangent axis 0 xyz, scale 0
  float4 a1;  // tangent axis 1 xyz, scale 1
  float4 e;   // reflectivity, opacity, -, -
};
static_assert(sizeof(Surfel) == 80, "Surfel layout");

// Internal node with both child boxes.  child >= 0: internal node index;
// child < 0: leaf ~child.
struct __align__(16) BvhNode {
  float4 b0;  // left lo x,y,z, left hi x
  float4 b1;  // left hi y,z, right lo x,y
  float4 b2;  // right lo z, right hi x,y,z
  int4 c;     // left child, right child, -, -
};
static_assert(sizeof(BvhNode) == 64, "BvhNode layout");

struct AccelHeader {
  int32_t surfel_count;  // planar surfels (device-computed)
  int32_t status;
  uint32_t bounds_bits[6];  // order-preserving encoded scene AABB of the means
  int64_t sort_counters[5]; // counters[1] = items to sort (raw-key onesweep)
};

struct AccelLayout {
  int64_t header;
  int64_t surfels;     // Surfel[G]
  int64_t semantics;   // int64[G]
  int64_t nodes;       // BvhNode[max(L-1,1)]
  int64_t parents;     // int32[2L]: parent of internal node i at [i], of leaf l at [L + l]
  int64_t flags;       // uint32[L]
  int64_t keys_a;      // uint64[G]
  int64_t keys_b;      // uint64[G]
  int64_t vals_a;      // int32[G]
  int64_t vals_b;      // int32[G]
  int64_t sort;        // ScratchLayout region
  ScratchLayout sort_layout;
  int64_t total;
};

AccelLayout make_accel_layout(int64_t count, int packet) {
  AccelLayout l{};
  const int64_t leaves = (count + packet - 1) / packet;
  int64_t off = 0;
  auto take = [&](int64_t bytes) {
    const int64_t at = off;
    off = align_up(off + bytes, 256);
    return at;
  };
  l.header = take(sizeof(AccelHeader));
  l.surfels = take(count * static_cast<int64_t>(sizeof(Surfel)));
  l.semantics = take(count * 8);
  l.nodes = take((leaves > 1 ? leaves - 1 : 1) * static_cast<int64_t>(sizeof(BvhNode)));
  l.parents = take(2 * (leaves > 0 ? leaves : 1) * 4);
  l.flags = take((leaves > 0 ? leaves : 1) * 4);
  l.keys_a = take(count * 8);
  l.keys_b = take(count * 8);
  l.vals_a = take(count * 4);
  l.vals_b = take(count * 4);
  l.sort_layout = make_scratch_layout(count > 0 ? count : 1, 0, true);
  l.sort = take(l.sort_layout.total);
  l.total = off;
  return l;
}

__device__ __forceinline__ void quaternion_axes(const float* q, float3 axes[3]) {
  const float w = q[0], x = q[1], y = q[2], z = q[3];
  axes[0] = make_float3(1.0f - 2.0f * (y * y + z * z), 2.0f * (x * y + z * w), 2.0f * (x * z - y * w));
  axes[1] = make_float3(2.0f * (x * y - z * w), 1.0f - 2.0f * (x * x + z * z), 2.0f * (y * z + x * w));
  axes[2] = make_float3(2.0f * (x * z + y * w), 2.0f * (y * z - x * w), 1.0f - 2.0f * (x * x + y * y));
}

__device__ __forceinline__ float comp(float3 v, int axis) {
  return axis == 0 ? v.x : (axis == 1 ? v.y : v.z);
}

__device__ __forceinline__ bool planar_axes(const float* scales, float planarity, int* normal_axis,
                                            int* t0, int* t1) {
  int n = 0;
  if (scales[1] < scales[n]) n = 1;
  if (scales[2] < scales[n]) n = 2;
  const int a = n == 0 ? 1 : 0;
  const int b = n == 2 ? 1 : 2;
  *normal_axis = n;
  *t0 = a;
  *t1 = b;
  const float tangent_min = fminf(scales[a], scales[b]);
  return scales[n] > 0.0f && !(scales[n] / tangent_min > planarity);
}

// ---------------------------------------------------------------- build
struct BuildParams {
  const float* means;
  const float* scales;
  const float* rotations;
  const float* opacities;
  const int64_t* semantics;
  const float* reflectivity;
  const float* confidence;
  int64_t count;
  int packet;
  float support_sigma;
  float planarity;
  unsigned char* accel;
  AccelLayout layout;
};

__global__ void __launch_bounds__(kLidarThreads) lidar_bounds_kernel(BuildParams p) {
  AccelHeader* h = reinterpret_cast<AccelHeader*>(p.accel + p.layout.header);
  uint32_t lo[3] = {0xffffffffu, 0xffffffffu, 0xffffffffu};
  uint32_t hi[3] = {0u, 0u, 0u};
  for (int64_t g = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; g < p.count;
       g += static_cast<int64_t>(gridDim.x) * blockDim.x) {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const uint32_t v = float_order(p.means[g * 3 + a]);
      lo[a] = min(lo[a], v);
      hi[a] = max(hi[a], v);
    }
  }
#pragma unroll
  for (int a = 0; a < 3; ++a) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      lo[a] = min(lo[a], __shfl_xor_sync(0xffffffffu, lo[a], o));
      hi[a] = max(hi[a], __shfl_xor_sync(0xffffffffu, hi[a], o));
    }
    if ((threadIdx.x & 31) == 0) {
      atomicMin(&h->bounds_bits[a], lo[a]);
      atomicMax(&h->bounds_bits[3 + a], hi[a]);
    }
  }
}

// Morton key of planar surfels (reference quantisation), kNonPlanarKey for
// the rest; value = Gaussian index; counts the planar surfels.
__global__ void __launch_bounds__(kLidarThreads) lidar_keys_kernel(BuildParams p) {
  AccelHeader* h = reinterpret_cast<AccelHeader*>(p.accel + p.layout.header);
  uint64_t* keys = reinterpret_cast<uint64_t*>(p.accel + p.layout.keys_a);
  int32_t* vals = reinterpret_cast<int32_t*>(p.accel + p.layout.vals_a);
  const int64_t g = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  bool planar = false;
  if (g < p.count) {
    int n, t0, t1;
    planar = planar_axes(p.scales + g * 3, p.planarity, &n, &t0, &t1);
    uint32_t key = kNonPlanarKey;
    if (planar) {
      uint32_t q[3];
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        const float low = order_float(h->bounds_bits[a]);
        const float extent = fmaxf(order_float(h->bounds_bits[3 + a]) - low, 1.0e-12f);
        const float normalized = fminf(fmaxf((p.means[g * 3 + a] - low) / extent, 0.0f), 1.0f);
        q[a] = static_cast<uint32_t>(normalized * 1023.0f + 0.5f);
      }
      key = expand_bits(q[0]) | (expand_bits(q[1]) << 1) | (expand_bits(q[2]) << 2);
    }
    keys[g] = key;
    vals[g] = static_cast<int32_t>(g);
  }
  const uint32_t planar_in_warp = __popc(__ballot_sync(0xffffffffu, planar));
  if ((threadIdx.x & 31) == 0 && planar_in_warp) atomicAdd(&h->surfel_count, planar_in_warp);
}

// Surfel records in Morton order.
__global__ void __launch_bounds__(kLidarThreads) lidar_gather_kernel(BuildParams p,
                                                                      const int32_t* sorted) {
  const AccelHeader* h = reinterpret_cast<const AccelHeader*>(p.accel + p.layout.header);
  Surfel* surfels = reinterpret_cast<Surfel*>(p.accel + p.layout.surfels);
  int64_t* sem = reinterpret_cast<int64_t*>(p.accel + p.layout.semantics);
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= h->surfel_count) return;
  const int64_t g = sorted[i];
  int n, t0, t1;
  const float* sc = p.scales + g * 3;
  planar_axes(sc, p.planarity, &n, &t0, &t1);
  float3 axes[3];
  quaternion_axes(p.rotations + g * 4, axes);
  Surfel s;
  const float smax = fmaxf(sc[t0], sc[t1]);
  s.m = make_float4(p.means[g * 3 + 0], p.means[g * 3 + 1], p.means[g * 3 + 2], smax * smax);
  s.n = make_float4(axes[n].x, axes[n].y, axes[n].z, p.confidence ? p.confidence[g] : 1.0f);
  s.a0 = make_float4(axes[t0].x, axes[t0].y, axes[t0].z, sc[t0]);
  s.a1 = make_float4(axes[t1].x, axes[t1].y, axes[t1].z, sc[t1]);
  s.e = make_float4(p.reflectivity ? p.reflectivity[g] : -1.0f, p.opacities[g], 0.0f, 0.0f);
  surfels[i] = s;
  sem[i] = p.semantics[g];
}

__device__ __forceinline__ uint64_t leaf_key(const uint64_t* morton, int leaf, int packet) {
  return (morton[static_cast<int64_t>(leaf) * packet] << 32) | static_cast<uint32_t>(leaf);
}

__device__ __forceinline__ int delta(const uint64_t* morton, int packet, int leaves, int i, int j) {
  if (j < 0 || j >= leaves) return -1;
  return __clzll(leaf_key(morton, i, packet) ^ leaf_key(morton, j, packet));
}

// Karras (2012) radix tree over the sorted leaf keys; internal node i's
// children are internal nodes or leaves (encoded ~leaf).
__global__ void __launch_bounds__(kLidarThreads) lidar_tree_kernel(BuildParams p,
                                                                    const uint64_t* morton) {
  const AccelHeader* h = reinterpret_cast<const AccelHeader*>(p.accel + p.layout.header);
  BvhNode* nodes = reinterpret_cast<BvhNode*>(p.accel + p.layout.nodes);
  int32_t* parents = reinterpret_cast<int32_t*>(p.accel + p.layout.parents);
  uint32_t* flags = reinterpret_cast<uint32_t*>(p.accel + p.layout.flags);
  const int m = h->surfel_count;
  const int leaves = (m + p.packet - 1) / p.packet;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < leaves) flags[i] = 0u;
  if (i >= leaves - 1) return;
  const int d = (delta(morton, p.packet, leaves, i, i + 1) - delta(morton, p.packet, leaves, i, i - 1)) >= 0 ? 1 : -1;
  const int dmin = delta(morton, p.packet, leaves, i, i - d);
  int lmax = 2;
  while (delta(morton, p.packet, leaves, i, i + lmax * d) > dmin) lmax <<= 1;
  int l = 0;
  for (int t = lmax >> 1; t >= 1; t >>= 1) {
    if (delta(morton, p.packet, leaves, i, i + (l + t) * d) > dmin) l += t;
  }
  const int j = i + l * d;
  const int dnode = delta(morton, p.packet, leaves, i, j);
  int s = 0;
  int t = l;
  do {
    t = (t + 1) >> 1;
    if (delta(morton, p.packet, leaves, i, i + (s + t) * d) > dnode) s += t;
  } while (t > 1);
  const int split = i + s * d + min(d, 0);
  const int lo = min(i, j);
  const int hi = max(i, j);
  const int left = (lo == split) ? ~split : split;
  const int right = (hi == split + 1) ? ~(split + 1) : (split + 1);
  nodes[i].c = make_int4(left, right, 0, 0);
  if (left >= 0) parents[left] = i; else parents[leaves + ~left] = i;
  if (right >= 0) parents[right] = i; else parents[leaves + ~right] = i;
  if (i == 0) parents[0] = -1;
}

// Leaf boxes (tangent-ellipse bounds, reference :195-256) and the bottom-up
// refit: a node's box union is computed by whichever child arrives second.
__global__ void __launch_bounds__(kLidarThreads) lidar_refit_kernel(BuildParams p) {
  const AccelHeader* h = reinterpret_cast<const AccelHeader*>(p.accel + p.layout.header);
  const Surfel* surfels = reinterpret_cast<const Surfel*>(p.accel + p.layout.surfels);
  BvhNode* nodes = reinterpret_cast<BvhNode*>(p.accel + p.layout.nodes);
  const int32_t* parents = reinterpret_cast<const int32_t*>(p.accel + p.layout.parents);
  uint32_t* flags = reinterpret_cast<uint32_t*>(p.accel + p.layout.flags);
  const int m = h->surfel_count;
  const int leaves = (m + p.packet - 1) / p.packet;
  const int leaf = blockIdx.x * blockDim.x + threadIdx.x;
  if (leaf >= leaves || leaves < 2) return;
  float lo[3] = {CUDART_INF_F, CUDART_INF_F, CUDART_INF_F};
  float hi[3] = {-CUDART_INF_F, -CUDART_INF_F, -CUDART_INF_F};
  const int begin = leaf * p.packet;
  const int end = min(begin + p.packet, m);
  for (int k = begin; k < end; ++k) {
    const Surfel s = surfels[k];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const float a0 = a == 0 ? s.a0.x : (a == 1 ? s.a0.y : s.a0.z);
      const float a1 = a == 0 ? s.a1.x : (a == 1 ? s.a1.y : s.a1.z);
      const float c = a == 0 ? s.m.x : (a == 1 ? s.m.y : s.m.z);
      const float extent = p.support_sigma * (fabsf(a0) * s.a0.w + fabsf(a1) * s.a1.w) + 1.0e-4f;
      lo[a] = fminf(lo[a], c - extent);
      hi[a] = fmaxf(hi[a], c + extent);
    }
  }
  int child = ~leaf;
  int node = parents[leaves + leaf];
  while (node >= 0) {
    BvhNode* n = nodes + node;
    const bool is_left = n->c.x == child;
    if (is_left) {
      n->b0 = make_float4(lo[0], lo[1], lo[2], hi[0]);
      n->b1.x = hi[1];
      n->b1.y = hi[2];
    } else {
      n->b1.z = lo[0];
      n->b1.w = lo[1];
      n->b2 = make_float4(lo[2], hi[0], hi[1], hi[2]);
    }
    __threadfence();
    if (atomicAdd(flags + node, 1u) == 0u) return;  // sibling not done yet
    __threadfence();
    const float4 b0 = __ldcg(&n->b0);
    const float4 b1 = __ldcg(&n->b1);
    const float4 b2 = __ldcg(&n->b2);
    lo[0] = fminf(b0.x, b1.z);
    lo[1] = fminf(b0.y, b1.w);
    lo[2] = fminf(b0.z, b2.x);
    hi[0] = fmaxf(b0.w, b2.y);
    hi[1] = fmaxf(b1.x, b2.z);
    hi[2] = fmaxf(b1.y, b2.w);
    child = node;
    node = parents[node];
  }
}

struct LidarDescriptor {
  int64_t scene_id;
  const Surfel* surfels;
  const int64_t* semantics;
  const BvhNode* nodes;
  const AccelHeader* header;
  int32_t packet;
  int32_t pad[17];
};
static_assert(sizeof(LidarDescriptor) == 14 * 8, "descriptor is one reference [S,14] int64 row");

__global__ void lidar_pack_kernel(LidarDescriptor* table, int64_t slot, LidarDescriptor d) {
  table[slot] = d;
}

// ---------------------------------------------------------------- trace
struct TraceParams {
  const LidarDescriptor* descriptors;
  int scene_count;
  const float* dirs;
  int64_t rays;
  const int32_t* times_i32;
  const int64_t* times_i64;
  const float* sensor_to_world;
  const float* scene_to_world;
  const int64_t* scene_ids;
  const int64_t* active;
  int64_t active_count;
  const int32_t* ray_order;  // [rays] trace order, or null
  int64_t batch;
  int returns;
  float near_plane, far_plane, q_max, threshold, min_cos, cluster_abs, cluster_rel;
  float fallback_reflectivity, dir_tol;
  int semantic_slots;
  float* range;
  float* position;
  float* intensity;
  int64_t* semantic;
  bool* valid;
  int64_t* time_out;
  int32_t* return_count;
  int64_t* counters;
};

enum : int {
  kCallsStarted = 0, kCallsCompleted, kRaysTraced, kNodeVisits, kLeafTests, kCandidates,
  kReturns, kStackOverflow, kSemanticOverflow, kInvalidDirections, kInvalidSceneIds,
  kInvalidActiveSensorIds,
};

__global__ void __launch_bounds__(kLidarThreads) lidar_clear_kernel(TraceParams p, int64_t total) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i == 0) atomicAdd(reinterpret_cast<unsigned long long*>(p.counters + kCallsStarted), 1ull);
  if (i >= total) return;
  p.range[i] = CUDART_INF_F;
  p.intensity[i] = 0.0f;
  p.semantic[i] = -1;
  p.valid[i] = false;
  p.position[3 * i + 0] = 0.0f;
  p.position[3 * i + 1] = 0.0f;
  p.position[3 * i + 2] = 0.0f;
  const int64_t ray = (i / p.returns) % p.rays;
  p.time_out[i] = p.times_i64 ? p.times_i64[ray] : static_cast<int64_t>(p.times_i32[ray]);
  if (i % p.returns == 0) p.return_count[i / p.returns] = 0;
}

__global__ void lidar_end_kernel(int64_t* counters) {
  atomicAdd(reinterpret_cast<unsigned long long*>(counters + kCallsCompleted), 1ull);
}

// Ray in the scene frame.  inv = 1/d per axis and ood = o * inv, so a slab
// bound is one fma; an axis with d == 0 gives infinite (or NaN) bounds, which
// the min/max below ignore, so such a box is kept (conservatively) rather
// than culled.  inv_dd = 1/|d|^2 for the surfel distance pre-test.
struct Ray {
  float3 o, d, inv, ood;
  float inv_dd;
};

// Slab test of one box against [tmin, tmax] (reference :329-363), branch
// free; empty boxes (lo > hi) never hit.  *entry = where the ray enters.
__device__ __forceinline__ bool hit_box(const Ray& r, float lx, float ly, float lz, float hx,
                                        float hy, float hz, float tmin, float tmax, float* entry) {
  const float ax = fmaf(lx, r.inv.x, -r.ood.x), bx = fmaf(hx, r.inv.x, -r.ood.x);
  const float ay = fmaf(ly, r.inv.y, -r.ood.y), by = fmaf(hy, r.inv.y, -r.ood.y);
  const float az = fmaf(lz, r.inv.z, -r.ood.z), bz = fmaf(hz, r.inv.z, -r.ood.z);
  const float t0 = fmaxf(fmaxf(tmin, fminf(ax, bx)), fmaxf(fminf(ay, by), fminf(az, bz)));
  const float t1 = fminf(fminf(tmax, fmaxf(ax, bx)), fminf(fmaxf(ay, by), fmaxf(az, bz)));
  *entry = t0;
  return t0 <= t1 && lx <= hx;
}

struct Candidate {
  float t, weight, intensity;
};

// Candidate test of one surfel (reference :383-421).  A conservative
// pre-test comes first: an accepted hit point lies in the surfel's tangent
// plane with tangent coordinates (u, v), u^2 + v^2 <= q_max, so within
// sqrt(q_max) * max(scale0, scale1) of the mean, and the ray must pass at
// least that close (distance from the cross product, which does not cancel).
// Only surfels that pass it load their frame and take the exact test.
__device__ __forceinline__ bool near_surfel(const float4& m, const Ray& r, const TraceParams& p) {
  const float3 dm = make_float3(m.x - r.o.x, m.y - r.o.y, m.z - r.o.z);
  const float cx = dm.y * r.d.z - dm.z * r.d.y;
  const float cy = dm.z * r.d.x - dm.x * r.d.z;
  const float cz = dm.x * r.d.y - dm.y * r.d.x;
  const float dist2 = (cx * cx + cy * cy + cz * cz) * r.inv_dd;
  return dist2 <= p.q_max * m.w * 1.001f + 1.0e-5f;
}

// The exact test of a surfel that passed near_surfel.
__device__ __forceinline__ bool evaluate_near(const Surfel* sp, const Ray& r, const TraceParams& p,
                                              Candidate* c) {
  const float4 m = __ldg(&sp->m);
  const float3 dm = make_float3(m.x - r.o.x, m.y - r.o.y, m.z - r.o.z);
  const float4 n = __ldg(&sp->n);
  const float denom = n.x * r.d.x + n.y * r.d.y + n.z * r.d.z;
  const float incidence = fabsf(denom);
  if (incidence < p.min_cos) return false;
  const float t = (n.x * dm.x + n.y * dm.y + n.z * dm.z) / denom;
  if (!(t >= p.near_plane && t <= p.far_plane)) return false;
  const float4 a0 = __ldg(&sp->a0);
  const float4 a1 = __ldg(&sp->a1);
  const float3 diff = make_float3(r.o.x + r.d.x * t - m.x, r.o.y + r.d.y * t - m.y,
                                  r.o.z + r.d.z * t - m.z);
  const float u = (diff.x * a0.x + diff.y * a0.y + diff.z * a0.z) / a0.w;
  const float v = (diff.x * a1.x + diff.y * a1.y + diff.z * a1.z) / a1.w;
  const float q = u * u + v * v;
  if (!(q <= p.q_max)) return false;
  const float support = expf(-0.5f * q);
  const float4 e = __ldg(&sp->e);
  const float weight = e.y * support * n.w;
  if (!(weight >= p.threshold) || !isfinite(weight)) return false;
  const float refl = e.x >= 0.0f ? e.x : p.fallback_reflectivity;
  c->t = t;
  c->weight = weight;
  c->intensity = fminf(fmaxf(refl * support * incidence, 0.0f), 1.0f);
  return true;
}

__device__ __forceinline__ bool evaluate(const Surfel* sp, const Ray& r, const TraceParams& p,
                                         Candidate* c) {
  return near_surfel(__ldg(&sp->m), r, p) && evaluate_near(sp, r, p, c);
}

struct TraceStats {
  uint32_t nodes, tests, candidates;
  bool overflow;
};

// Visits the leaves whose boxes the ray crosses inside [tmin, *tmax], nearest
// box first; visit(leaf) may shrink *tmax, which prunes deferred entries.
//
// Warp-coherent: the lanes that reach this call with the same hierarchy walk
// it together.  The stack of node codes is the same for all of them (every
// push is decided by ballots), each lane keeps its own entry distances and a
// bit per entry saying whether its own ray hit that box, and each lane still
// tests, prunes and visits exactly the boxes its own ray crosses - so every
// ray gets the leaves it would get alone, while the warp runs one loop
// instead of up to 32 divergent ones (coherent rays of a scan share most of
// their nodes).  Children hit by several lanes are ordered by the majority's
// nearer child.
// The node-code and lane-mask stacks of a warp whose 32 lanes traverse one
// hierarchy together live in shared memory (the entries are the same in
// every lane, and every lane writes the same values, so no lane can read a
// slot another lane has not finished writing); each lane's entry distances
// stay in its own local array.  A partial group keeps all three locally.
__shared__ int s_trace_stack[kTraceThreads / 32][kMaxStack];
__shared__ uint32_t s_trace_lanes[kTraceThreads / 32][kMaxStack];

template <typename Visit>
__device__ __forceinline__ void traverse_walk(const LidarDescriptor& sc, const Ray& r, float tmin,
                                              float* tmax, TraceStats& st, Visit& visit,
                                              unsigned group, int* stack, uint32_t* lanes) {
  const int lane = threadIdx.x & 31;
  float entry[kMaxStack];
  int top = 0;
  // The entry to process next is held in registers (the root first, then
  // the nearer child of each node): only the farther child of a node whose
  // two children are both hit goes through the stack.  The order of visits
  // is the one of a stack that pushes the nearer child last.
  int code = 0;
  uint32_t held = group;
  float held_entry = tmin;
  bool have = true;
  const float kInf = __int_as_float(0x7f800000);
  while (true) {  // top, code, held, stack[] and lanes[] are the same in every lane of the group
    if (!have) {
      if (top == 0) break;
      --top;
      code = stack[top];
      held = lanes[top];
      held_entry = entry[top];
    }
    have = false;
    const bool mine = ((held >> lane) & 1u) != 0u && held_entry <= *tmax;
    if (code < 0) {
      if (mine) visit(~code);
      continue;
    }
    if (!__any_sync(group, mine)) continue;
    const BvhNode* node = sc.nodes + code;
    const int4 kids = __ldg(&node->c);  // the same node for every lane of the group
    float el = kInf, er = kInf;
    bool hl = false, hr = false;
    if (mine) {
      ++st.nodes;
      const float4 b0 = __ldg(&node->b0), b1 = __ldg(&node->b1), b2 = __ldg(&node->b2);
      hl = hit_box(r, b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, tmin, *tmax, &el);
      hr = hit_box(r, b1.z, b1.w, b2.x, b2.y, b2.z, b2.w, tmin, *tmax, &er);
      if (!hl) el = kInf;
      if (!hr) er = kInf;
    }
    const unsigned ml = __ballot_sync(group, hl);
    const unsigned mr = __ballot_sync(group, hr);
    const unsigned left_first = __ballot_sync(group, hl && hr && el <= er);
    if (ml != 0u && mr != 0u) {
      if (top + 1 > kMaxStack) {
        st.overflow = true;
        return;
      }
      const bool left_near = 2 * __popc(left_first) >= __popc(ml & mr);
      stack[top] = left_near ? kids.y : kids.x;
      lanes[top] = left_near ? mr : ml;
      entry[top] = left_near ? er : el;
      ++top;
      code = left_near ? kids.x : kids.y;
      held = left_near ? ml : mr;
      held_entry = left_near ? el : er;
      have = true;
    } else if (ml != 0u) {
      code = kids.x;
      held = ml;
      held_entry = el;
      have = true;
    } else if (mr != 0u) {
      code = kids.y;
      held = mr;
      held_entry = er;
      have = true;
    }
  }
}

template <bool kWarpStack, typename Visit>
__device__ __forceinline__ void traverse(const LidarDescriptor& sc, int leaves, const Ray& r,
                                         float tmin, float* tmax, TraceStats& st, Visit visit) {
  if (leaves <= 0) return;
  if (leaves == 1) {
    ++st.nodes;
    visit(0);
    return;
  }
  const unsigned group =
      __match_any_sync(__activemask(), reinterpret_cast<unsigned long long>(sc.nodes));
  if (kWarpStack && group == 0xffffffffu) {
    const int warp = threadIdx.x >> 5;
    traverse_walk(sc, r, tmin, tmax, st, visit, group, s_trace_stack[warp], s_trace_lanes[warp]);
  } else {
    int stack[kMaxStack];
    uint32_t lanes[kMaxStack];
    traverse_walk(sc, r, tmin, tmax, st, visit, group, stack, lanes);
  }
}

__device__ __forceinline__ void add_counter(int64_t* counters, int index, uint32_t value) {
  // Warp-aggregated counter update.
  const uint32_t total = __reduce_add_sync(0xffffffffu, value);
  if ((threadIdx.x & 31) == 0 && total) {
    atomicAdd(reinterpret_cast<unsigned long long*>(counters + index),
              static_cast<unsigned long long>(total));
  }
}

// Two-warp CTAs, eighteen resident per SM (1,152 threads and a 56-register
// cap, some spills to L1): the traversal is latency-bound, and extra warps
// pay for some spills (per 16.8M-ray frame in ray-direction order: 20 / 18
// CTAs per SM at 48 / 56 registers measured 13.6 / 13.3 ms, and 24 at 40
// registers 9 % slower than 20; in the given ray order, 256-thread CTAs at
// 4 / 5 / 6 / 8 per SM measured 24.5 / 22.3 / 23.2 / 24.9 ms).  Ray costs vary a lot (hits,
// misses, grazing rays), and a CTA keeps its slot until its slowest warp is
// done: small CTAs free their slots at a finer grain, while the hardware
// scheduler still hands out consecutive rays, which share most of their
// nodes.
__global__ void __launch_bounds__(kTraceThreads, 18) lidar_trace_kernel(TraceParams p) {
  const int64_t work = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const int64_t total = p.active_count * p.rays;
  uint32_t traced = 0, bad_dir = 0, bad_scene = 0, bad_active = 0, returns_found = 0;
  uint32_t sem_overflow = 0, stack_overflow = 0;
  TraceStats st{0u, 0u, 0u, false};
  if (work < total) {
    const int64_t a = work / p.rays;
    const int64_t local = work - a * p.rays;
    const int64_t ray = p.ray_order ? static_cast<int64_t>(p.ray_order[local]) : local;
    int64_t sensor = p.active ? p.active[a] : a;
    bool ok = true;
    if (ray < 0 || ray >= p.rays) {
      bad_dir = 1u;  // a ray order that is not a permutation
      ok = false;
    } else if (p.active && a > 0 && sensor <= p.active[a - 1]) {
      bad_active = ray == 0 ? 1u : 0u;
      ok = false;
    } else if (sensor < 0 || sensor >= p.batch) {
      bad_active = 1u;
      ok = false;
    }
    const LidarDescriptor* scene = nullptr;
    if (ok) {
      traced = 1u;
      const float dx = p.dirs[ray * 3 + 0], dy = p.dirs[ray * 3 + 1], dz = p.dirs[ray * 3 + 2];
      const float norm2 = dx * dx + dy * dy + dz * dz;
      const float lower = 1.0f - p.dir_tol, upper = 1.0f + p.dir_tol;
      if (!isfinite(norm2) || norm2 < lower * lower || norm2 > upper * upper) {
        bad_dir = 1u;
        ok = false;
      }
      if (ok) {
        const int64_t sid = p.scene_ids[sensor];
        for (int k = 0; k < p.scene_count; ++k) {
          if (p.descriptors[k].scene_id == sid) {
            scene = p.descriptors + k;
            break;
          }
        }
        if (!scene) {
          bad_scene = 1u;
          ok = false;
        }
      }
      if (ok) {
        const float* st_m = p.sensor_to_world + 16 * sensor;
        const float3 wo = make_float3(st_m[3], st_m[7], st_m[11]);
        const float3 wd = make_float3(st_m[0] * dx + st_m[1] * dy + st_m[2] * dz,
                                      st_m[4] * dx + st_m[5] * dy + st_m[6] * dz,
                                      st_m[8] * dx + st_m[9] * dy + st_m[10] * dz);
        const float* xt = p.scene_to_world + 16 * sensor;
        const float3 tr = make_float3(wo.x - xt[3], wo.y - xt[7], wo.z - xt[11]);
        Ray r;
        r.o = make_float3(xt[0] * tr.x + xt[4] * tr.y + xt[8] * tr.z,
                          xt[1] * tr.x + xt[5] * tr.y + xt[9] * tr.z,
                          xt[2] * tr.x + xt[6] * tr.y + xt[10] * tr.z);
        r.d = make_float3(xt[0] * wd.x + xt[4] * wd.y + xt[8] * wd.z,
                          xt[1] * wd.x + xt[5] * wd.y + xt[9] * wd.z,
                          xt[2] * wd.x + xt[6] * wd.y + xt[10] * wd.z);
        r.inv = make_float3(1.0f / r.d.x, 1.0f / r.d.y, 1.0f / r.d.z);
        r.ood = make_float3(r.o.x * r.inv.x, r.o.y * r.inv.y, r.o.z * r.inv.z);
        r.inv_dd = 1.0f / (r.d.x * r.d.x + r.d.y * r.d.y + r.d.z * r.d.z);
        const LidarDescriptor sc = *scene;
        const int m = sc.header->surfel_count;
        const int leaves = (m + sc.packet - 1) / sc.packet;
        float previous_end = p.near_plane - 1.0e-6f;
        const int64_t base = (sensor * p.rays + ray) * p.returns;
        for (int k = 0; k < p.returns; ++k) {
          // One traversal finds the nearest candidate beyond the previous
          // cluster and keeps the candidates inside its cluster window
          // [best, best + max(abs, rel * best)]: the window only shrinks as
          // best does, so nodes beyond the current window are pruned and a
          // candidate dropped from the list can never re-enter the final
          // window.  If more than kMaxCluster candidates fall inside the
          // window at once, a second traversal gathers the cluster.
          float best = p.far_plane;
          float window = p.far_plane;
          bool found = false;
          int listed = 0;
          bool list_full = false;
          int32_t list_idx[kMaxCluster];
          float list_t[kMaxCluster];
          traverse<true>(sc, leaves, r, p.near_plane, &window, st, [&](int leaf) {
            const int begin = leaf * sc.packet;
            const int end = min(begin + sc.packet, m);
            // Distance pre-tests of the whole leaf first, so that its
            // surfels' loads are in flight together.
            uint32_t near = 0u;
#pragma unroll 4
            for (int i = begin; i < end; ++i) {
              near |= near_surfel(__ldg(&sc.surfels[i].m), r, p) ? 1u << (i - begin) : 0u;
            }
            st.tests += static_cast<uint32_t>(end - begin);
            while (near) {
              const int i = begin + __ffs(near) - 1;
              near &= near - 1u;
              Candidate c;
              if (!evaluate_near(sc.surfels + i, r, p, &c)) continue;
              ++st.candidates;
              if (!(c.t > previous_end) || c.t > window) continue;
              if (!found || c.t < best) {
                best = c.t;
                found = true;
                window = fminf(p.far_plane, best + fmaxf(p.cluster_abs, p.cluster_rel * best));
                int kept = 0;
                for (int q = 0; q < listed; ++q) {
                  if (list_t[q] <= window) {
                    list_t[kept] = list_t[q];
                    list_idx[kept] = list_idx[q];
                    ++kept;
                  }
                }
                listed = kept;
              }
              if (listed < kMaxCluster) {
                list_t[listed] = c.t;
                list_idx[listed] = i;
                ++listed;
              } else {
                list_full = true;
              }
            }
          });
          if (st.overflow || !found) break;
          const float first_t = best;
          const float cluster_end = window;
          // Cluster reduction in double precision.
          int64_t labels[kMaxSemanticSlots];
          double label_w[kMaxSemanticSlots];
          int nl = 0;
          bool overflow = false;
          double total_w = 0.0, weighted_t = 0.0, weighted_i = 0.0;
          auto accumulate = [&](int i, const Candidate& c) {
            total_w += static_cast<double>(c.weight);
            weighted_t += static_cast<double>(c.weight) * c.t;
            weighted_i += static_cast<double>(c.weight) * c.intensity;
            const int64_t label = sc.semantics[i];
            int slot = -1;
            for (int q = 0; q < nl; ++q) {
              if (labels[q] == label) {
                slot = q;
                break;
              }
            }
            if (slot < 0) {
              if (nl >= p.semantic_slots) {
                overflow = true;
              } else {
                slot = nl++;
                labels[slot] = label;
                label_w[slot] = 0.0;
              }
            }
            if (slot >= 0) label_w[slot] += static_cast<double>(c.weight);
          };
          if (!list_full) {
            for (int q = 0; q < listed; ++q) {
              Candidate c;
              if (evaluate(sc.surfels + list_idx[q], r, p, &c)) accumulate(list_idx[q], c);
            }
          } else {
            float window_end = cluster_end;
            traverse<false>(sc, leaves, r, first_t, &window_end, st, [&](int leaf) {
              const int begin = leaf * sc.packet;
              const int end = min(begin + sc.packet, m);
              for (int i = begin; i < end; ++i) {
                ++st.tests;
                Candidate c;
                if (!evaluate(sc.surfels + i, r, p, &c) || c.t < first_t || c.t > cluster_end) continue;
                accumulate(i, c);
              }
            });
          }
          if (st.overflow) break;
          if (overflow) {
            sem_overflow = 1u;
            break;
          }
          if (!(total_w > 0.0)) break;
          int win = 0;
          for (int q = 1; q < nl; ++q) {
            if (label_w[q] > label_w[win] || (label_w[q] == label_w[win] && labels[q] < labels[win])) {
              win = q;
            }
          }
          const float range = static_cast<float>(weighted_t / total_w);
          const int64_t out = base + k;
          p.range[out] = range;
          p.intensity[out] = static_cast<float>(weighted_i / total_w);
          p.semantic[out] = labels[win];
          p.valid[out] = true;
          p.position[3 * out + 0] = wo.x + wd.x * range;
          p.position[3 * out + 1] = wo.y + wd.y * range;
          p.position[3 * out + 2] = wo.z + wd.z * range;
          ++returns_found;
          previous_end = cluster_end;
        }
        p.return_count[sensor * p.rays + ray] = static_cast<int32_t>(returns_found);
        stack_overflow = st.overflow ? 1u : 0u;
      }
    }
  }
  add_counter(p.counters, kRaysTraced, traced);
  add_counter(p.counters, kNodeVisits, st.nodes);
  add_counter(p.counters, kLeafTests, st.tests);
  add_counter(p.counters, kCandidates, st.candidates);
  add_counter(p.counters, kReturns, returns_found);
  add_counter(p.counters, kStackOverflow, stack_overflow);
  add_counter(p.counters, kSemanticOverflow, sem_overflow);
  add_counter(p.counters, kInvalidDirections, bad_dir);
  add_counter(p.counters, kInvalidSceneIds, bad_scene);
  add_counter(p.counters, kInvalidActiveSensorIds, bad_active);
}

}  // namespace
}  // namespace vgr

// ---------------------------------------------------------------- C ABI
namespace vgr {
namespace {

__global__ void lidar_init_kernel(unsigned char* accel, AccelLayout layout, int64_t count) {
  AccelHeader* h = reinterpret_cast<AccelHeader*>(accel + layout.header);
  h->surfel_count = 0;
  h->status = 0;
  for (int a = 0; a < 3; ++a) {
    h->bounds_bits[a] = 0xffffffffu;
    h->bounds_bits[3 + a] = 0u;
  }
  for (int k = 0; k < 5; ++k) h->sort_counters[k] = 0;
  h->sort_counters[1] = count;
  ScratchHeader* sh = reinterpret_cast<ScratchHeader*>(accel + layout.sort + layout.sort_layout.header);
  uint32_t* words = reinterpret_cast<uint32_t*>(sh);
  for (int k = 0; k < 32; ++k) words[k] = 0u;
  uint32_t* hist = reinterpret_cast<uint32_t*>(accel + layout.sort + layout.sort_layout.sort_hist);
  for (int k = 0; k < kMaxSortPasses * kRadixBins; ++k) hist[k] = 0u;
}

unsigned grid_for(int64_t items, int threads) {
  const int64_t blocks = (items + threads - 1) / threads;
  return static_cast<unsigned>(blocks < 1 ? 1 : blocks);
}

}  // namespace
}  // namespace vgr

using namespace vgr;

extern "C" int64_t vgr_lidar_sort_temp_bytes(int64_t num_items, int32_t packet_size) {
  if (num_items <= 0) return fail(VGR_ERR_INVALID_ARGUMENT, "num_items must be positive");
  if (num_items > INT_MAX) return fail(VGR_ERR_INVALID_ARGUMENT, "at most INT_MAX Gaussians per scene");
  if (packet_size != 8 && packet_size != 16) {
    return fail(VGR_ERR_INVALID_ARGUMENT, "packet_size must be 8 or 16");
  }
  return make_accel_layout(num_items, packet_size).total;
}

extern "C" int vgr_lidar_build_scene_lbvh(const vgr_lidar_scene* scene, int32_t packet_size,
                                          double support_sigma, double planarity_ratio_max,
                                          void* accel, int64_t accel_bytes, void* stream_ptr) {
  if (!scene || !accel) return fail(VGR_ERR_INVALID_ARGUMENT, "scene and accel must be non-null");
  if (packet_size != 8 && packet_size != 16) {
    return fail(VGR_ERR_INVALID_ARGUMENT, "packet_size must be 8 or 16");
  }
  if (!(support_sigma > 0.0)) return fail(VGR_ERR_INVALID_ARGUMENT, "support_sigma must be positive");
  if (!(planarity_ratio_max > 0.0 && planarity_ratio_max <= 1.0)) {
    return fail(VGR_ERR_INVALID_ARGUMENT, "planarity_ratio_max must be in (0, 1]");
  }
  if (scene->count <= 0 || scene->count > INT_MAX) {
    return fail(VGR_ERR_INVALID_ARGUMENT, "a LiDAR scene needs 1..INT_MAX Gaussians");
  }
  if (!scene->means || !scene->scales || !scene->rotations || !scene->opacities ||
      !scene->semantic_ids) {
    return fail(VGR_ERR_INVALID_ARGUMENT, "scene tensors must be non-null");
  }
  if ((reinterpret_cast<uintptr_t>(accel) & 255) != 0) {
    return fail(VGR_ERR_INVALID_ARGUMENT, "accel buffer must be 256-byte aligned");
  }
  const AccelLayout layout = make_accel_layout(scene->count, packet_size);
  if (accel_bytes < layout.total) {
    return fail(VGR_ERR_SCRATCH_TOO_SMALL, "LiDAR accel buffer holds %lld bytes, needs %lld",
                static_cast<long long>(accel_bytes), static_cast<long long>(layout.total));
  }
  int sms = 0;
  int rc = device_sms(&sms);
  if (rc != VGR_OK) return rc;
  cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
  unsigned char* base = static_cast<unsigned char*>(accel);
  BuildParams bp{};
  bp.means = scene->means;
  bp.scales = scene->scales;
  bp.rotations = scene->rotations;
  bp.opacities = scene->opacities;
  bp.semantics = scene->semantic_ids;
  bp.reflectivity = scene->reflectivity;
  bp.confidence = scene->surface_confidence;
  bp.count = scene->count;
  bp.packet = packet_size;
  bp.support_sigma = static_cast<float>(support_sigma);
  bp.planarity = static_cast<float>(planarity_ratio_max);
  bp.accel = base;
  bp.layout = layout;

  lidar_init_kernel<<<1, 1, 0, stream>>>(base, layout, scene->count);
  if ((rc = check_launch("lidar build: init")) != VGR_OK) return rc;
  const unsigned bgrid = grid_for(scene->count, kLidarThreads) < static_cast<unsigned>(sms * 4)
                             ? grid_for(scene->count, kLidarThreads)
                             : static_cast<unsigned>(sms * 4);
  lidar_bounds_kernel<<<bgrid, kLidarThreads, 0, stream>>>(bp);
  if ((rc = check_launch("lidar build: bounds")) != VGR_OK) return rc;
  lidar_keys_kernel<<<grid_for(scene->count, kLidarThreads), kLidarThreads, 0, stream>>>(bp);
  if ((rc = check_launch("lidar build: keys")) != VGR_OK) return rc;

  // Stable raw-key radix sort of 31-bit keys (Morton | non-planar flag).
  SortParams so{};
  so.scratch = base + layout.sort;
  so.layout = layout.sort_layout;
  so.counters = reinterpret_cast<const int64_t*>(base + layout.header + offsetof(AccelHeader, sort_counters));
  so.capacity = scene->count;
  so.map.raw = 1;
  so.map.total_bits = 31;
  so.passes = 4;
  so.keys_in = reinterpret_cast<uint64_t*>(base + layout.keys_a);
  const int64_t parts = layout.sort_layout.max_partitions;
  sort_histogram_kernel<<<static_cast<unsigned>(parts < sms * 4 ? parts : sms * 4), kSortThreads, 0,
                          stream>>>(so);
  if ((rc = check_launch("lidar build: sort histogram")) != VGR_OK) return rc;
  uint64_t* kin = reinterpret_cast<uint64_t*>(base + layout.keys_a);
  uint64_t* kout = reinterpret_cast<uint64_t*>(base + layout.keys_b);
  int32_t* vin = reinterpret_cast<int32_t*>(base + layout.vals_a);
  int32_t* vout = reinterpret_cast<int32_t*>(base + layout.vals_b);
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
    if ((rc = check_launch("lidar build: sort pass")) != VGR_OK) return rc;
    uint64_t* tk = kin; kin = kout; kout = tk;
    int32_t* tv = vin; vin = vout; vout = tv;
  }
  lidar_gather_kernel<<<grid_for(scene->count, kLidarThreads), kLidarThreads, 0, stream>>>(bp, vin);
  if ((rc = check_launch("lidar build: gather")) != VGR_OK) return rc;
  const int64_t max_leaves = (scene->count + packet_size - 1) / packet_size;
  lidar_tree_kernel<<<grid_for(max_leaves, kLidarThreads), kLidarThreads, 0, stream>>>(bp, kin);
  if ((rc = check_launch("lidar build: tree")) != VGR_OK) return rc;
  lidar_refit_kernel<<<grid_for(max_leaves, kLidarThreads), kLidarThreads, 0, stream>>>(bp);
  return check_launch("lidar build: refit");
}

extern "C" int vgr_lidar_pack_scene_descriptor(void* descriptors, int64_t descriptor_capacity,
                                               int64_t slot, int64_t scene_id, const void* accel,
                                               int64_t gaussian_count, int32_t packet_size,
                                               void* stream) {
  if (!descriptors || !accel) return fail(VGR_ERR_INVALID_ARGUMENT, "descriptors and accel must be non-null");
  if (slot < 0 || slot >= descriptor_capacity) {
    return fail(VGR_ERR_INVALID_ARGUMENT, "descriptor slot out of range");
  }
  if (packet_size != 8 && packet_size != 16) {
    return fail(VGR_ERR_INVALID_ARGUMENT, "packet_size must be 8 or 16");
  }
  if (gaussian_count <= 0) return fail(VGR_ERR_INVALID_ARGUMENT, "invalid leaf metadata");
  const AccelLayout layout = make_accel_layout(gaussian_count, packet_size);
  const unsigned char* base = static_cast<const unsigned char*>(accel);
  LidarDescriptor d{};
  d.scene_id = scene_id;
  d.surfels = reinterpret_cast<const Surfel*>(base + layout.surfels);
  d.semantics = reinterpret_cast<const int64_t*>(base + layout.semantics);
  d.nodes = reinterpret_cast<const BvhNode*>(base + layout.nodes);
  d.header = reinterpret_cast<const AccelHeader*>(base + layout.header);
  d.packet = packet_size;
  lidar_pack_kernel<<<1, 1, 0, static_cast<cudaStream_t>(stream)>>>(
      static_cast<LidarDescriptor*>(descriptors), slot, d);
  return check_launch("lidar pack descriptor");
}

extern "C" int vgr_render_lidar(const void* descriptors, int64_t scene_count,
                                const vgr_lidar_inputs* in, const vgr_lidar_outputs* out,
                                int64_t* counters, const vgr_lidar_options* opt,
                                void* stream_ptr) {
  if (!descriptors || !in || !out || !counters || !opt) {
    return fail(VGR_ERR_INVALID_ARGUMENT, "render_lidar arguments must be non-null");
  }
  if (scene_count <= 0) return fail(VGR_ERR_INVALID_ARGUMENT, "invalid scene_count");
  if (opt->returns != 1 && opt->returns != 2) return fail(VGR_ERR_INVALID_ARGUMENT, "returns must be 1 or 2");
  if (!(opt->near_plane_m > 0.0 && opt->far_plane_m > opt->near_plane_m)) {
    return fail(VGR_ERR_INVALID_ARGUMENT, "invalid range planes");
  }
  if (!(opt->support_sigma > 0.0)) return fail(VGR_ERR_INVALID_ARGUMENT, "support_sigma must be positive");
  if (!(opt->detection_threshold > 0.0 && opt->detection_threshold <= 1.0)) {
    return fail(VGR_ERR_INVALID_ARGUMENT, "invalid threshold");
  }
  if (!(opt->min_incidence_cos > 0.0 && opt->min_incidence_cos <= 1.0)) {
    return fail(VGR_ERR_INVALID_ARGUMENT, "invalid incidence");
  }
  if (!(opt->cluster_abs_m >= 0.0 && opt->cluster_relative >= 0.0)) {
    return fail(VGR_ERR_INVALID_ARGUMENT, "invalid cluster");
  }
  if (!(opt->fallback_reflectivity >= 0.0 && opt->fallback_reflectivity <= 1.0)) {
    return fail(VGR_ERR_INVALID_ARGUMENT, "invalid reflectivity");
  }
  if (!(opt->direction_norm_tolerance > 0.0 && opt->direction_norm_tolerance < 1.0)) {
    return fail(VGR_ERR_INVALID_ARGUMENT, "direction tolerance must be in (0, 1)");
  }
  if (opt->semantic_slots <= 0 || opt->semantic_slots > 32) {
    return fail(VGR_ERR_INVALID_ARGUMENT, "semantic_slots must be in [1, 32]");
  }
  if (in->rays <= 0 || in->batch <= 0 || in->rays > INT_MAX || in->batch > INT_MAX) {
    return fail(VGR_ERR_INVALID_ARGUMENT, "rays and batch must be in [1, INT_MAX]");
  }
  if (!in->ray_directions || !in->time_offsets || !in->sensor_to_world || !in->scene_to_world ||
      !in->scene_ids) {
    return fail(VGR_ERR_INVALID_ARGUMENT, "LiDAR inputs must be non-null");
  }
  if (!out->range_m || !out->position_world_m || !out->intensity || !out->semantic_id ||
      !out->valid || !out->time_offset_ns || !out->return_count) {
    return fail(VGR_ERR_INVALID_ARGUMENT, "LiDAR outputs must be non-null");
  }
  cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
  TraceParams tp{};
  tp.descriptors = static_cast<const LidarDescriptor*>(descriptors);
  tp.scene_count = static_cast<int>(scene_count);
  tp.dirs = in->ray_directions;
  tp.rays = in->rays;
  tp.ray_order = in->ray_order;
  tp.times_i64 = in->time_offsets_are_int64 ? static_cast<const int64_t*>(in->time_offsets) : nullptr;
  tp.times_i32 = in->time_offsets_are_int64 ? nullptr : static_cast<const int32_t*>(in->time_offsets);
  tp.sensor_to_world = in->sensor_to_world;
  tp.scene_to_world = in->scene_to_world;
  tp.scene_ids = in->scene_ids;
  tp.active = in->active_sensor_ids;
  tp.active_count = in->active_sensor_ids ? in->active_count : in->batch;
  tp.batch = in->batch;
  tp.returns = opt->returns;
  tp.near_plane = static_cast<float>(opt->near_plane_m);
  tp.far_plane = static_cast<float>(opt->far_plane_m);
  tp.q_max = static_cast<float>(opt->support_sigma * opt->support_sigma);
  tp.threshold = static_cast<float>(opt->detection_threshold);
  tp.min_cos = static_cast<float>(opt->min_incidence_cos);
  tp.cluster_abs = static_cast<float>(opt->cluster_abs_m);
  tp.cluster_rel = static_cast<float>(opt->cluster_relative);
  tp.fallback_reflectivity = static_cast<float>(opt->fallback_reflectivity);
  tp.dir_tol = static_cast<float>(opt->direction_norm_tolerance);
  tp.semantic_slots = opt->semantic_slots;
  tp.range = out->range_m;
  tp.position = out->position_world_m;
  tp.intensity = out->intensity;
  tp.semantic = out->semantic_id;
  tp.valid = reinterpret_cast<bool*>(out->valid);
  tp.time_out = out->time_offset_ns;
  tp.return_count = out->return_count;
  tp.counters = counters;
  const int64_t total_returns = in->batch * in->rays * opt->returns;
  lidar_clear_kernel<<<grid_for(total_returns, kLidarThreads), kLidarThreads, 0, stream>>>(
      tp, total_returns);
  int rc = check_launch("render_lidar: clear");
  if (rc != VGR_OK) return rc;
  const int64_t work = tp.active_count * in->rays;
  if (work > 0) {
    lidar_trace_kernel<<<grid_for(work, kTraceThreads), kTraceThreads, 0, stream>>>(tp);
    if ((rc = check_launch("render_lidar: trace")) != VGR_OK) return rc;
  }
  lidar_end_kernel<<<1, 1, 0, stream>>>(counters);
  return check_launch("render_lidar: end");
}
