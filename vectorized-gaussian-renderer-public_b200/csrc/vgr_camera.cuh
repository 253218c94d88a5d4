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

// Scratch header at offset 0 of the scratch buffer.
struct ScratchHeader {
  int32_t status;              // device error bits (kDeviceError*)
  int32_t pad0;
  uint32_t project_queue;      // virtual-block ticket of the projection kernel
  uint32_t composite_queue;    // work-item ticket of the persistent compositor
  uint32_t sort_queue[8];      // partition ticket per radix pass (LBVH sort)
  uint32_t ranges_done;
  uint32_t bucket_total;       // keys placed in tile buckets (tile_scan_kernel)
  uint32_t tail_cursor;        // overflow-sentinel keys placed after the buckets
  uint32_t pad1;
  unsigned long long visible_total;  // records reserved by the projection blocks
  unsigned long long isect_total;    // keys reserved by the projection blocks
  uint32_t pad2[12];
};
static_assert(sizeof(ScratchHeader) == 128, "ScratchHeader layout");

constexpr int kProjectThreads = 256;
constexpr int kProjectRounds = 2;
constexpr int kProjectChunk = kProjectThreads * kProjectRounds;  // tasks per virtual block

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
constexpr int kTileScanThreads = 1024;
constexpr int kTileScanItems = 16;


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
