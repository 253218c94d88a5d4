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
};

__global__ void camera_setup_kernel(SetupParams p);
template <int kShDegree>
__global__ void project_emit_kernel(ProjectParams p);
__global__ void sort_histogram_kernel(SortParams p);
__global__ void sort_onesweep_kernel(SortParams p);
__global__ void tile_scan_kernel(BucketParams p);
__global__ void bucket_scatter_kernel(BucketParams p);
__global__ void tile_sort_kernel(BucketParams p);
template <int kTile, bool kFull>
__global__ void composite_kernel(CompositeParams p);

// Threads per compositor CTA (two pixels per thread, 8x8-pixel warp blocks).
constexpr int composite_threads(int tile) { return tile >= 16 ? 128 : 32; }

}  // namespace vgr
