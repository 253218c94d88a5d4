// Internal data layout shared by the camera-path kernels.
#pragma once

#include <cuda_fp16.h>
#include <stdint.h>

#include "vgr_common.cuh"

namespace vgr {

// Per active camera slot, built on the device by camera_setup_kernel.
struct CamPlan {
  int32_t camera;       // index into the batch, -1 when the active id is invalid
  int32_t scene_slot;   // registered scene slot, -1 when unregistered
  int64_t g_begin;      // first packed Gaussian of the camera's scene
  int64_t g_count;      // Gaussians in the scene (0 when unregistered)
  int32_t width;
  int32_t height;
  int32_t tiles_x;
  int32_t tiles_y;
  int64_t tile_base;    // global tile id of the camera's tile (0,0)
  int64_t pixel_base;   // first output pixel of the camera
};
static_assert(sizeof(CamPlan) == 56, "CamPlan layout");

// Projected record, three float4 (VGR_RECORD_BYTES = 48).
struct __align__(16) Record {
  float4 a;  // mean_x, mean_y, conic_xx, conic_xy
  float4 b;  // conic_yy, opacity, depth, bits(gaussian id)
  float4 c;  // red, green, blue, bits(half2(hx, hy))
};

// ---------------------------------------------------------------------------
// Per-camera constants of the projection, computed once per active slot by
// the setup kernel.  R = view_rotation * env_rotation and
// t = view_rotation * env_t + view_t, so camera-space p = R m + t.
// ---------------------------------------------------------------------------
struct __align__(16) CamConst {
  float r[9];
  float t[3];
  float fx, fy, cx, cy;
  float lim_xp, lim_xn, lim_yp, lim_yn;
  float width, height;
  float r_scale2;   // upper bound of the largest eigenvalue of R^T R (1 for a rotation)
  float pad[3];
};
static_assert(sizeof(CamConst) == 112, "CamConst is fourteen 8-byte words");

__device__ __forceinline__ void make_cam_const(const float* view, const float* env,
                                               const float* intr, int width, int height,
                                               CamConst* c) {
#pragma unroll
  for (int row = 0; row < 3; ++row) {
#pragma unroll
    for (int col = 0; col < 3; ++col) {
      c->r[row * 3 + col] =
          ffma(view[row * 4 + 2], env[8 + col],
               ffma(view[row * 4 + 1], env[4 + col], fmul(view[row * 4 + 0], env[col])));
    }
    c->t[row] = ffma(view[row * 4 + 2], env[11],
                     ffma(view[row * 4 + 1], env[7],
                          ffma(view[row * 4 + 0], env[3], view[row * 4 + 3])));
  }
  c->fx = intr[0];
  c->fy = intr[4];
  c->cx = intr[2];
  c->cy = intr[5];
  const float w = static_cast<float>(width);
  const float h = static_cast<float>(height);
  c->width = w;
  c->height = h;
  const float tan_x = fdiv(fmul(0.5f, w), c->fx);
  const float tan_y = fdiv(fmul(0.5f, h), c->fy);
  c->lim_xp = ffma(0.3f, tan_x, fdiv(fsub(w, c->cx), c->fx));
  c->lim_xn = ffma(0.3f, tan_x, fdiv(c->cx, c->fx));
  c->lim_yp = ffma(0.3f, tan_y, fdiv(fsub(h, c->cy), c->fy));
  c->lim_yn = ffma(0.3f, tan_y, fdiv(c->cy, c->fy));
  // Gershgorin bound of R^T R (R includes any scale of the object->world
  // transform); used only by the conservative early cull.
  float bound = 0.0f;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    float row = 0.0f;
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      const float m = c->r[i] * c->r[j] + c->r[3 + i] * c->r[3 + j] + c->r[6 + i] * c->r[6 + j];
      row += fabsf(m);
    }
    bound = fmaxf(bound, row);
  }
  c->r_scale2 = bound * 1.001f;
  c->pad[0] = c->pad[1] = c->pad[2] = 0.0f;
}

// Rotation matrix (row-major) of a WXYZ quaternion normalised by
// 1/sqrt(max(|q|^2, 1e-20)) with IEEE division and square root
// (renderer_cuda.cu:112-143); inv_norm receives that factor.
__device__ __forceinline__ void quaternion_rotation(float w, float x, float y, float z, float* r,
                                                    float* inv_norm) {
  const float norm2 = ffma(z, z, ffma(y, y, ffma(x, x, fmul(w, w))));
  const float inv = fdiv(1.0f, fsqrt(fmaxf(norm2, 1.0e-20f)));
  *inv_norm = inv;
  w = fmul(w, inv);
  x = fmul(x, inv);
  y = fmul(y, inv);
  z = fmul(z, inv);
  const float xx = fmul(x, x), yy = fmul(y, y), zz = fmul(z, z);
  const float xy = fmul(x, y), xz = fmul(x, z), yz = fmul(y, z);
  const float wx = fmul(w, x), wy = fmul(w, y), wz = fmul(w, z);
  r[0] = fsub(1.0f, fmul(2.0f, fadd(yy, zz)));
  r[1] = fmul(2.0f, fsub(xy, wz));
  r[2] = fmul(2.0f, fadd(xz, wy));
  r[3] = fmul(2.0f, fadd(xy, wz));
  r[4] = fsub(1.0f, fmul(2.0f, fadd(xx, zz)));
  r[5] = fmul(2.0f, fsub(yz, wx));
  r[6] = fmul(2.0f, fsub(xz, wy));
  r[7] = fmul(2.0f, fadd(yz, wx));
  r[8] = fsub(1.0f, fmul(2.0f, fadd(xx, yy)));
}

// Object-space covariance Sigma = R diag(s^2) R^T, upper triangle
// (00, 01, 02, 11, 12, 22) (renderer_cuda.cu:492-540).
__device__ __forceinline__ void covariance_from_quaternion(float w, float x, float y, float z,
                                                           float sx, float sy, float sz,
                                                           float* cov) {
  float r[9];
  float inv;
  quaternion_rotation(w, x, y, z, r, &inv);
  const float s2[3] = {fmul(sx, sx), fmul(sy, sy), fmul(sz, sz)};
  const int rows[6][2] = {{0, 0}, {0, 1}, {0, 2}, {1, 1}, {1, 2}, {2, 2}};
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    const float* a = r + rows[k][0] * 3;
    const float* b = r + rows[k][1] * 3;
    cov[k] =
        ffma(fmul(a[2], b[2]), s2[2], ffma(fmul(a[1], b[1]), s2[1], fmul(fmul(a[0], b[0]), s2[0])));
  }
}

// Scratch header at offset 0 of the scratch buffer.
struct ScratchHeader {
  int32_t status;              // device error bits (kDeviceError*)
  int32_t pad0;
  uint32_t project_queue;      // virtual-block ticket of the projection kernel
  uint32_t composite_queue;    // work-item ticket of the persistent compositor
  uint32_t sort_queue[8];      // partition ticket per radix pass (LBVH sort)
  uint32_t ranges_done;
  uint32_t bucket_total;       // keys placed in tile buckets (tile_span_scan_kernel)
  uint32_t tail_cursor;        // overflow-sentinel keys placed after the buckets
  uint32_t active_tiles;       // tiles with at least one key (tile_span_sum_kernel)
  unsigned long long visible_total;  // records reserved by the projection blocks
  unsigned long long isect_total;    // keys reserved by the projection blocks
  uint32_t large_tile_queue;         // tile ticket of the tile sort's large-bucket workers
  uint32_t large_tile_count;         // tiles listed for the large-bucket workers
  uint32_t pad2[10];
};
static_assert(sizeof(ScratchHeader) == 128, "ScratchHeader layout");

constexpr int kProjectThreads = 256;
constexpr int kProjectRounds = 2;
constexpr int kProjectChunk = kProjectThreads * kProjectRounds;  // tasks per virtual block
// A warp-round of the projection: the unit of the cluster cull.
constexpr int kProjectCluster = 32;
constexpr int kProjectClusters = kProjectChunk / kProjectCluster;  // clusters per chunk
static_assert(kProjectClusters <= 32, "one bit per cluster in a 32-bit mask");
constexpr int kTicketBatch = 32;  // virtual blocks taken per queue ticket (one per lane)
constexpr int kOwnerKeys = 2048;  // keys per block whose owners the projection tabulates

constexpr int kSortThreads = 256;
constexpr int kSortItems = 16;
constexpr int kSortTile = kSortThreads * kSortItems;  // keys per partition
constexpr int kRadixBits = 8;
constexpr int kRadixBins = 1 << kRadixBits;
// Dynamic shared memory of one onesweep CTA: the partition's keys and values.
constexpr int kSortDynamicSmem = kSortTile * (8 + 4);
constexpr int kMaxSortPasses = 8;

// Tile-bucket sort: one CTA per tile orders the tile's (depth, record) pairs
// in shared memory when they fit (kTileSortCap), else in chunks through global
// memory.
constexpr int kTileSortThreads = 256;
constexpr int kTileSortItems = 12;
constexpr int kTileSortCap = kTileSortThreads * kTileSortItems;
constexpr int kTileSortSplitBits = 11;  // depth-range splits of one bucket
constexpr int kTileScanThreads = 1024;
constexpr int kTileScanItems = 16;
// Tile scan in three passes: spans of kTileScanSpan tiles, one CTA each.
constexpr int kTileSpanThreads = 256;
constexpr int kTileScanSpan = kTileSpanThreads * kTileScanItems;


__host__ __device__ inline int64_t align_up(int64_t v, int64_t a) {
  return (v + a - 1) / a * a;
}

// Byte offsets of the scratch regions (all 256-byte aligned).
struct ScratchLayout {
  int64_t header;         // ScratchHeader
  int64_t plans;          // CamPlan[A]
  int64_t cam_consts;     // CamConst[A] (112 bytes each)
  int64_t tile_prefix;    // int64[A+1] exclusive prefix of tiles over active slots
  int64_t sort_hist;      // uint32[passes][256]
  int64_t sort_desc;      // uint64[passes][partitions][256]
  int64_t total;
  int64_t max_partitions;
};

// onesweep_descriptors: reserve the per-partition look-back descriptors of
// the global onesweep sort (the LBVH Morton sort); the camera path sorts in
// tile buckets and needs none.
__host__ __device__ inline ScratchLayout make_scratch_layout(
    int64_t intersection_capacity, int64_t max_active_cameras, bool onesweep_descriptors) {
  ScratchLayout l{};
  int64_t off = 0;
  l.header = off;
  off = align_up(off + static_cast<int64_t>(sizeof(ScratchHeader)), 256);
  l.plans = off;
  off = align_up(off + max_active_cameras * static_cast<int64_t>(sizeof(CamPlan)), 256);
  l.cam_consts = off;
  off = align_up(off + max_active_cameras * 112, 256);
  l.tile_prefix = off;
  off = align_up(off + (max_active_cameras + 1) * 8, 256);
  l.sort_hist = off;
  off = align_up(off + kMaxSortPasses * kRadixBins * 4, 256);
  l.sort_desc = off;
  l.max_partitions =
      onesweep_descriptors ? (intersection_capacity + kSortTile - 1) / kSortTile : 0;
  off = align_up(off + static_cast<int64_t>(kMaxSortPasses) * l.max_partitions * kRadixBins * 8, 256);
  l.total = off;
  return l;
}

// Composite digit function of the sort.  Keys keep the reference format
// (global_tile << 32 | float bits of depth); the sort orders them by
// (tile, depth_bits - near_bits), which spans tile_bits + depth_bits bits and
// is order-equivalent because every emitted depth lies in [near, far].
// Keys whose tile is out of range (overflow sentinels) map to all-ones.
struct SortKeyMap {
  uint32_t near_bits;
  uint32_t depth_bits;   // bit width of (far_bits - near_bits)
  uint32_t total_bits;   // tile bits + depth bits
  uint32_t tile_count;   // global tiles
  uint32_t raw;          // nonzero: digits come from the key itself (LBVH Morton sort)
};

__device__ __forceinline__ uint64_t composite_key(uint64_t key, const SortKeyMap& m) {
  if (m.raw) return key;
  const uint32_t tile = static_cast<uint32_t>(key >> 32);
  if (tile >= m.tile_count) {
    return ~0ull;
  }
  const uint32_t d = static_cast<uint32_t>(key) - m.near_bits;
  return (static_cast<uint64_t>(tile) << m.depth_bits) | d;
}

}  // namespace vgr
