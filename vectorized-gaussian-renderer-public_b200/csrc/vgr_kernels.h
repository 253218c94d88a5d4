// Kernel parameter blocks and kernel declarations of the camera path.
#pragma once

#include <stdint.h>

#include "vgr_camera.cuh"

namespace vgr {

struct SetupParams {
  unsigned char* scratch;
  ScratchLayout layout;
  int64_t* counters;
  int reset_counters;
  const int64_t* active_ids;
  int64_t active_count;
  int64_t batch;
  const int64_t* camera_scene_ids;
  const int64_t* registered_scene_ids;
  const int64_t* scene_offsets;
  int scene_count;
  const int32_t* widths;
  const int32_t* heights;
  const int64_t* tile_offsets;
  const int64_t* pixel_offsets;
  int width;
  int height;
  int tile_size;
  const float* viewmats;
  const float* intrinsics;
  const float* env_xforms;
};

struct ProjectParams {
  unsigned char* scratch;
  ScratchLayout layout;
  const float* means;
  const float* covariances;
  const float* opacities;
  const float* features;
  int64_t feature_width;
  bool vector_feature_loads;  // rows 16-byte aligned and a multiple of 4 floats
  bool wide_feature_loads;    // rows 32-byte aligned and a multiple of 8 floats
  const float* viewmats;
  const float* intrinsics;
  const float* env_xforms;
  int64_t active_count;
  int64_t total_vblocks;
  float near_plane;
  float far_plane;
  float support_sigma;
  float cov_eps;
  bool antialiased;
  int tile_size;
  void* records;
  int64_t visible_capacity;
  uint64_t* keys;
  int32_t* values;
  int64_t intersection_capacity;
  uint32_t* tile_counts;       // per-tile key counts (zeroed before the launch)
  int64_t tile_count;
  int64_t* counters;
  float* mirror_means2d;
  float* mirror_conics;
  float* mirror_depths;
  float* mirror_opacities;
  int32_t* mirror_camera_ids;
  int32_t* mirror_gaussian_ids;
  int32_t* mirror_radii;
  float* mirror_ray_precisions;       // exact-ray mode: [V,6] or null
  float* mirror_ray_precision_means;  // exact-ray mode: [V,4] or null
  int32_t* record_map;         // training: [A, record_map_stride] record of (slot, local Gaussian)
  int64_t record_map_stride;
  const int32_t* gaussian_ids; // reported id of packed Gaussian g, or null (g itself)
  const float4* chunk_bounds;  // [C,2] per-chunk bounds, or null (no chunk culling)
  const int64_t* chunk_offsets;// [S+1] first chunk of each registered scene
  const float4* cluster_bounds;// [C*kProjectClusters,2] per-cluster bounds, or null
  float4* ray_ext;             // exact-ray mode: [V,3] extension records, else null
  // Dense mode (optical-thickness depth cutoff).
  float* depth_tau;            // [B * sub-tiles, kDenseBuckets] optical-thickness lower bounds
  const int32_t* tile_cutoff;  // [T] last depth bucket a tile can still blend
  uint32_t near_bits;          // float bits of near_plane (bucket origin)
  int sub_x, sub_y;            // sub-tile grid of one image (kDenseSubtile pixels)
};

// Projection kernel variants: the plain fused projection + emission, and the
// two passes of dense mode (accumulate per-tile optical thickness by depth
// bucket; then project again and emit only keys in front of each tile's
// cutoff).
enum ProjectMode : int { kProjectPlain = 0, kProjectDenseTau = 1, kProjectDenseCull = 2 };

// Dense mode depth buckets: a monotone integer map of the depth's float bits,
// 16 buckets per octave above near_plane (bits >> 19), clamped to 256.
constexpr int kDenseBuckets = 256;
constexpr int kDenseSubtile = 4;  // pixels per side of the optical-thickness cells
constexpr float kDenseMinAlpha = 0.25f;  // cells below this alpha bound add nothing
constexpr int kDenseBucketShift = 19;
__device__ __forceinline__ int dense_bucket(float depth, uint32_t near_bits) {
  const uint32_t bits = __float_as_uint(depth);
  const uint32_t d = bits > near_bits ? (bits - near_bits) >> kDenseBucketShift : 0u;
  return d < static_cast<uint32_t>(kDenseBuckets) ? static_cast<int>(d) : kDenseBuckets - 1;
}

struct DenseCutoffParams {
  unsigned char* scratch;
  ScratchLayout layout;
  const float* depth_tau;      // [B * sub_x * sub_y, kDenseBuckets]
  int32_t* tile_cutoff;        // [T], zeroed before the launch
  int64_t sub_count;           // B * sub_x * sub_y
  int sub_x, sub_y;            // sub-tiles per image row / column
  int tiles_x;                 // tiles per image row
  int64_t tiles_per_image;
  int tile_size;               // pixels per tile side (a multiple of kDenseSubtile)
};

struct SortParams {
  unsigned char* scratch;
  ScratchLayout layout;
  const int64_t* counters;     // counters[1] = emitted keys
  int64_t capacity;
  SortKeyMap map;
  int passes;
  int pass;
  const uint64_t* keys_in;
  const int32_t* values_in;
  uint64_t* keys_out;
  int32_t* values_out;
};


// Tile-bucket sort of the emitted intersections.  tile_ends holds per-tile
// key counts after projection, then scatter cursors, then range ends.
struct BucketParams {
  unsigned char* scratch;
  ScratchLayout layout;
  int64_t* counters;           // [1] emitted keys in, [4] active tiles out
  int64_t capacity;            // intersection capacity
  int64_t tile_count;          // global tiles
  const uint64_t* keys_in;     // emission order: tile << 32 | depth bits
  const int32_t* values_in;    // record index per key
  uint64_t* keys_out;          // bucketed (depth bits | record << 32), then sorted keys
  int32_t* values_out;         // sorted record indices
  uint64_t* temp;              // ping-pong space for tiles above kTileSortCap
  int32_t* tile_starts;
  int32_t* tile_ends;
  const Record* records;       // projected records (Gaussian ids break depth ties)
  int64_t visible_capacity;
  int64_t large_workers;       // tile sort: leading CTAs that sort the buckets above kTileSortCap
  int32_t* large_list;         // tiles above kTileSortCap (in the consumed values_in buffer)
};

struct CompositeParams {
  unsigned char* scratch;
  ScratchLayout layout;
  int64_t active_count;
  int64_t tiles_per_camera_hint;  // >0 when every camera has this many tiles
  const Record* records;
  const int32_t* values;
  const int32_t* tile_starts;
  const int32_t* tile_ends;
  const int64_t* semantic_ids;
  float semantic_min_alpha;
  bool output_srgb;
  float* rgb;
  float* depth;
  float* alpha;
  int64_t* semantic;
  float* final_transmittance;  // training: [P] transmittance after the last blended record
  int32_t* last_position;      // training: [P] sorted position one past the last blended record
  bool persistent;             // resident grid over a device work queue
  // Exact-ray mode.
  const float4* ray_ext;       // [V,3] (P00,P01,P02,P11), (P12,P22,Pm0,Pm1), (Pm2,mPm,-,-)
  const float* intrinsics;     // [B,3,3]
  float support_sigma;
};

template <int kTile, int kPix = 2>
struct CompositeGeometry {
  static_assert(kPix == 1 || kPix == 2, "one or two pixels per thread");
  static constexpr int kBlockW = kTile < 8 ? kTile : 8;  // warp block width (px)
  static constexpr int kLaneRows =
      (32 / kBlockW) < (kTile / kPix) ? (32 / kBlockW) : (kTile / kPix);  // lane rows
  static constexpr int kBlockH = kPix * kLaneRows;  // warp block height (px)
  static constexpr int kWarpsX = kTile / kBlockW;
  static constexpr int kWarpsY = kTile / kBlockH;
  static constexpr int kWarps = kWarpsX * kWarpsY;
  static constexpr int kThreads = kWarps * 32;
};

// Compositor CTA shapes (vgr_render_options.composite_shape): the default
// two pixels per thread at the tuned occupancy; one pixel per thread (8x4
// warp blocks, twice the threads, finer warp masks); two pixels per thread
// at half occupancy (no register spills).
constexpr int kShapeDefault = 0;
constexpr int kShapeOnePixel = 1;
constexpr int kShapeHalfOccupancy = 2;
template <int kShape>
struct CompositeShape {
  static constexpr int kPix = kShape == kShapeOnePixel ? 1 : 2;
};

constexpr int kCompositeBatch = 256;

// Shared-memory form of one record for the compositor loops (forward and
// backward use the same values, so both see the same alpha decisions):
// geo = (mean_x, mean_y, -conic_xx/2, -conic_xy), cpo = (-conic_yy/2, lo,
// opacity, -), col = (r, g, b, depth), and the mask of the warp blocks the
// record's conservative alpha footprint touches.  lo = max(-qmax/2, -20)
// merges the footprint bound with the reference's power >= -20 cut.
template <int kTile, int kPix = 2>
__device__ __forceinline__ void stage_composite_record(const Record& rec, float tile_x0,
                                                       float tile_y0, float4& geo, float4& cpo,
                                                       float4& col, uint32_t& mask_out) {
  using Geo = CompositeGeometry<kTile, kPix>;
  geo = make_float4(rec.a.x, rec.a.y, fmul(-0.5f, rec.a.z), -rec.a.w);
  const float o = rec.b.y;
  const float qmax = fminf(40.0f, 2.0f * __logf(255.0f * o)) * 1.001f + 1.0e-3f;
  cpo = make_float4(fmul(-0.5f, rec.b.x), fmaxf(fmul(-0.5f, qmax), -20.0f), o, 0.0f);
  col = make_float4(rec.c.x, rec.c.y, rec.c.z, rec.b.z);
  const __half2 box = *reinterpret_cast<const __half2*>(&rec.c.w);
  const float hx = __low2float(box);
  const float hy = __high2float(box);
  uint32_t mask = 0;
#pragma unroll
  for (int w = 0; w < Geo::kWarps; ++w) {
    const float bx0 = tile_x0 + static_cast<float>((w % Geo::kWarpsX) * Geo::kBlockW) + 0.5f;
    const float by0 = tile_y0 + static_cast<float>((w / Geo::kWarpsX) * Geo::kBlockH) + 0.5f;
    const float bx1 = bx0 + static_cast<float>(Geo::kBlockW - 1);
    const float by1 = by0 + static_cast<float>(Geo::kBlockH - 1);
    const bool hit = rec.a.x + hx >= bx0 && rec.a.x - hx <= bx1 && rec.a.y + hy >= by0 &&
                     rec.a.y - hy <= by1;
    mask |= hit ? (1u << w) : 0u;
  }
  mask_out = mask;
}

// Work item (one (camera, tile) of the compositor grid) -> active slot plan
// and tile index within the camera.  Slots are dense in [0, A) and every
// slot's tiles are contiguous; tile_prefix is monotone, so it is searched
// (starting from item / hint when every camera has `hint` tiles).
__device__ __forceinline__ bool locate_tile(const unsigned char* scratch, const ScratchLayout& layout,
                                            int64_t active_count, int64_t hint, int64_t item,
                                            CamPlan& plan, int64_t& local_tile) {
  const CamPlan* plans = reinterpret_cast<const CamPlan*>(scratch + layout.plans);
  const int64_t* tile_prefix = reinterpret_cast<const int64_t*>(scratch + layout.tile_prefix);
  const int64_t total = tile_prefix[active_count];
  if (item >= total) return false;
  int64_t lo = 0, hi = active_count;  // tile_prefix[lo] <= item < tile_prefix[hi]
  if (hint > 0) {
    const int64_t guess = item / hint;
    if (guess < active_count && tile_prefix[guess] <= item && item < tile_prefix[guess + 1]) {
      lo = guess;
      hi = guess + 1;
    }
  }
  while (hi - lo > 1) {
    const int64_t mid = (lo + hi) >> 1;
    if (tile_prefix[mid] <= item) lo = mid; else hi = mid;
  }
  plan = plans[lo];
  local_tile = item - tile_prefix[lo];
  return true;
}

// Differentiable form.
struct TrainActivateParams {
  const float* log_scales;      // [G,3]
  const float* rotations;       // [G,4] WXYZ, any norm
  const float* opacity_logits;  // [G]
  int64_t count;
  float* covariances;           // [G,6] out
  float* opacities;             // [G] out
};

struct CompositeBackwardParams {
  const unsigned char* scratch;
  ScratchLayout layout;
  int64_t active_count;
  int64_t tiles_per_camera_hint;
  const Record* records;
  const int32_t* values;              // sorted record indices
  const int32_t* tile_starts;
  const int32_t* tile_ends;
  const float* final_transmittance;   // [P]
  const int32_t* last_position;       // [P]
  const float* depth;                 // [P] forward depth output
  const float* grad_rgb;              // [P,3]
  const float* grad_depth;            // [P] or null
  const float* grad_alpha;            // [P] or null
  float4* record_grads;               // [V,3]
};

struct PhotometricLossParams {
  const float* rgb;            // [P,3]
  const float* target_rgb;     // [P,3]
  const float* depth;          // [P]
  const float* target_depth;   // [P]
  int64_t pixels;
  float depth_weight;
  float* loss;                 // [1], zeroed before the launch
  float* grad_rgb;             // [P,3] dL/drgb
  float* grad_depth;           // [P] dL/ddepth
};

struct ProjectBackwardParams {
  const unsigned char* scratch;
  ScratchLayout layout;
  int64_t active_count;
  const int64_t* scene_offsets;
  int scene_count;
  int64_t gaussian_count;
  const float* means;
  const float* covariances;     // forward activation output
  const float* opacities;       // forward activation output
  const float* features;
  int64_t feature_width;
  bool vector_feature_loads;    // rows 16-byte aligned and a multiple of 4 floats
  const float* log_scales;
  const float* rotations;
  float cov_eps;
  const int32_t* record_map;
  int64_t record_map_stride;
  const float4* record_grads;
  float* d_means;
  float* d_log_scales;
  float* d_rotations;
  float* d_opacity_logits;
  float* d_features;
};

__global__ void camera_setup_kernel(SetupParams p);
template <int kShDegree, bool kRay, int kMode>
__global__ void project_emit_kernel(ProjectParams p);
__global__ void dense_cutoff_kernel(DenseCutoffParams p);
__global__ void sort_histogram_kernel(SortParams p);
__global__ void sort_onesweep_kernel(SortParams p);
__global__ void tile_span_sum_kernel(BucketParams p);
__global__ void tile_span_scan_kernel(BucketParams p, int64_t spans);
__global__ void tile_span_apply_kernel(BucketParams p);
__global__ void bucket_scatter_kernel(BucketParams p);
__global__ void large_tile_list_kernel(BucketParams p);
__global__ void tile_sort_kernel(BucketParams p);
template <int kTile, bool kFull, bool kTrain, int kSplit, int kShape>
__global__ void composite_kernel(CompositeParams p);
template <int kTile, bool kFull, int kSplit>
__global__ void composite_ray_kernel(CompositeParams p);

__global__ void train_activate_kernel(TrainActivateParams p);
__global__ void zero_record_grads_kernel(float4* grads, const int64_t* counters, int64_t capacity);
__global__ void photometric_loss_kernel(PhotometricLossParams p);
template <int kTile>
__global__ void composite_backward_kernel(CompositeBackwardParams p);
template <int kShDegree>
__global__ void project_backward_kernel(ProjectBackwardParams p);

// Threads per compositor CTA (two pixels per thread, 8x8-pixel warp blocks).
constexpr int composite_threads(int tile) { return tile >= 32 ? 512 : tile >= 16 ? 128 : 32; }

}  // namespace vgr
