// C ABI of the camera path (declared in include/vgr_b200.h).
//
// Validation mirrors the TORCH_CHECKs of the reference binding
// (src/isaacsim_gaussian_renderer/native/renderer.cpp:214-310 and
// renderer_cuda.cu:2561-2730); violations return VGR_ERR_INVALID_ARGUMENT with
// the reference's message text in vgr_last_error().
#include <cuda_runtime.h>

#include <atomic>
#include <climits>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>

#include "../../include/vgr_b200.h"
#include "vgr_api_internal.h"
#include "vgr_kernels.h"
#include "vgr_misc.h"

namespace {

thread_local char g_last_error[1024] = "";
std::atomic<int64_t> g_launch_count{0};

struct OccupancyCache {
  int device = -1;
  int sms = 0;
  int project_blocks = 0;
};
thread_local OccupancyCache g_occ;

}  // namespace

static_assert(vgr::kProjectChunk == VGR_PROJECT_CHUNK, "projection chunk of the C ABI");
static_assert(vgr::kProjectCluster == VGR_PROJECT_CLUSTER, "projection cluster of the C ABI");
static_assert(vgr::kDenseBuckets == VGR_DENSE_DEPTH_BUCKETS, "dense depth buckets of the C ABI");
static_assert(vgr::kDenseSubtile == VGR_DENSE_CELL, "dense optical-thickness cell of the C ABI");

namespace vgr {

int fail(int code, const char* fmt, ...) {
  va_list args;
  va_start(args, fmt);
  std::vsnprintf(g_last_error, sizeof(g_last_error), fmt, args);
  va_end(args);
  return code;
}

int check_launch(const char* what, int launches) {
  g_launch_count.fetch_add(launches, std::memory_order_relaxed);
  const cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) {
    return fail(VGR_ERR_CUDA, "%s: %s", what, cudaGetErrorString(err));
  }
  return VGR_OK;
}

int device_sms(int* sms) {
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess) return fail(VGR_ERR_CUDA, "cudaGetDevice failed");
  if (g_occ.device != device) {
    g_occ = OccupancyCache{};
    g_occ.device = device;
    if (cudaDeviceGetAttribute(&g_occ.sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) {
      return fail(VGR_ERR_CUDA, "cudaDeviceGetAttribute(MultiProcessorCount) failed");
    }
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&g_occ.project_blocks, project_emit_kernel<3, false, kProjectPlain>,
                                                  kProjectThreads, 0);
    // The onesweep partition (LBVH Morton sort) needs more than the default
    // 48 KB of dynamic shared memory.
    cudaFuncSetAttribute(sort_onesweep_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         kSortDynamicSmem);
    if (g_occ.project_blocks < 1) g_occ.project_blocks = 1;
    cudaGetLastError();
  }
  *sms = g_occ.sms;
  return VGR_OK;
}

int64_t render_vblocks(int64_t active, int64_t max_scene_gaussians) {
  return active * ((max_scene_gaussians + kProjectChunk - 1) / kProjectChunk);
}

}  // namespace vgr

using namespace vgr;

extern "C" const char* vgr_version(void) { return "vgr_b200 0.1.0 sm_100a"; }

extern "C" const char* vgr_last_error(void) { return g_last_error; }

extern "C" int64_t vgr_kernel_launch_count(void) { return g_launch_count.load(); }
extern "C" int64_t vgr_project_chunk(void) { return kProjectChunk; }

extern "C" int64_t vgr_render_scratch_bytes(int64_t intersection_capacity,
                                            int64_t max_projection_tasks, int64_t global_tiles,
                                            int64_t max_active_cameras) {
  if (intersection_capacity <= 0 || max_projection_tasks < 0 || global_tiles <= 0 ||
      max_active_cameras < 0) {
    return fail(VGR_ERR_INVALID_ARGUMENT,
                "scratch query needs positive capacity and tile count, non-negative bounds");
  }
  return make_scratch_layout(intersection_capacity, max_active_cameras, false).total;
}

// Scratch for a drop-in caller that only knows (items, segments): active
// cameras are bounded by the tile count, projection tasks by 64 per item,
// and the visible records (one per item at most) are carved from the end.
static int64_t adapter_scratch_bytes(int64_t num_items, int64_t num_segments) {
  if (num_items <= 0) return fail(VGR_ERR_INVALID_ARGUMENT, "num_items must be positive");
  if (num_segments <= 0) return fail(VGR_ERR_INVALID_ARGUMENT, "num_segments must be positive");
  if (num_items > INT_MAX) {
    return fail(VGR_ERR_INVALID_ARGUMENT,
                "The first renderer implementation supports at most INT_MAX intersections");
  }
  if (num_segments > INT_MAX) {
    return fail(VGR_ERR_INVALID_ARGUMENT,
                "The first renderer implementation supports at most INT_MAX tile segments");
  }
  const int64_t active = num_segments < (1 << 20) ? num_segments : (1 << 20);
  const int64_t base = vgr_render_scratch_bytes(num_items, 64 * num_items, num_segments, active);
  return align_up(base, 256) + num_items * VGR_RECORD_BYTES;
}

extern "C" int64_t vgr_sort_temp_bytes(int64_t num_items, int64_t num_segments) {
  return adapter_scratch_bytes(num_items, num_segments);
}

extern "C" int64_t vgr_radix_sort_double_buffer_temp_bytes(int64_t num_items,
                                                           int64_t num_segments) {
  return adapter_scratch_bytes(num_items, num_segments);
}

extern "C" int vgr_precompute_covariances(const float* scales, const float* rotations,
                                          int64_t gaussian_count, float* covariances,
                                          void* stream) {
  if (gaussian_count < 0) return fail(VGR_ERR_INVALID_ARGUMENT, "gaussian count must be >= 0");
  if (gaussian_count == 0) return VGR_OK;
  if (!scales || !rotations || !covariances) {
    return fail(VGR_ERR_INVALID_ARGUMENT, "scales, rotations, and covariances must be non-null");
  }
  const int64_t blocks = (gaussian_count + 255) / 256;
  if (blocks > INT_MAX) return fail(VGR_ERR_INVALID_ARGUMENT, "covariance precompute grid exceeds CUDA limit");
  precompute_covariances_kernel<<<static_cast<unsigned>(blocks), 256, 0,
                                  static_cast<cudaStream_t>(stream)>>>(scales, rotations,
                                                                       gaussian_count, covariances);
  return check_launch("precompute_covariances");
}

extern "C" int vgr_prepare_chunked_active_ids(const int64_t* active_camera_ids,
                                              int64_t active_count, int32_t* active_mask,
                                              int64_t active_mask_capacity,
                                              int64_t* chunk_active_ids, int64_t chunk_rows,
                                              int64_t chunk_columns, int64_t logical_batch,
                                              int64_t physical_batch, void* stream) {
  if (logical_batch <= 0 || physical_batch <= 0) {
    return fail(VGR_ERR_INVALID_ARGUMENT, "logical and physical batches must be positive");
  }
  const int64_t chunk_count = (logical_batch + physical_batch - 1) / physical_batch;
  if (active_mask_capacity < logical_batch) {
    return fail(VGR_ERR_INVALID_ARGUMENT, "active_mask is too small for the logical batch");
  }
  if (chunk_rows < chunk_count || chunk_columns < physical_batch) {
    return fail(VGR_ERR_INVALID_ARGUMENT, "chunk_active_ids is too small for the chunk schedule");
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (cudaMemsetAsync(active_mask, 0, static_cast<size_t>(logical_batch) * sizeof(int32_t), s) !=
      cudaSuccess) {
    return check_launch("prepare_chunked_active_ids memset", 0);
  }
  if (active_count > 0) {
    const int64_t blocks = (active_count + 255) / 256;
    mark_active_kernel<<<static_cast<unsigned>(blocks), 256, 0, s>>>(active_camera_ids, active_count,
                                                                     active_mask, logical_batch);
  }
  const int64_t slots = chunk_count * physical_batch;
  build_chunk_ids_kernel<<<static_cast<unsigned>((slots + 255) / 256), 256, 0, s>>>(
      active_mask, logical_batch, physical_batch, slots, chunk_columns, chunk_active_ids);
  return check_launch("prepare_chunked_active_ids", active_count > 0 ? 2 : 1);
}

extern "C" int vgr_aggregate_chunk_counters(const int64_t* chunk_counters, int64_t chunk_rows,
                                            int64_t chunk_stride, int64_t* counters,
                                            int64_t* physical_capacity_counters,
                                            int64_t chunk_count, void* stream) {
  if (chunk_stride < 5) {
    return fail(VGR_ERR_INVALID_ARGUMENT,
                "chunk counters must have shape [N, >=5] and outputs >=5");
  }
  if (chunk_count <= 0 || chunk_count > chunk_rows) {
    return fail(VGR_ERR_INVALID_ARGUMENT, "chunk_count exceeds the counter workspace");
  }
  aggregate_counters_kernel<<<1, 32, 0, static_cast<cudaStream_t>(stream)>>>(
      chunk_counters, chunk_stride, chunk_count, counters, physical_capacity_counters);
  return check_launch("aggregate_chunk_counters");
}

namespace vgr {

// One CTA per work item, or a resident grid (as many CTAs as fit on the SMs)
// over the device work queue.
// kSplit > 1: each (kSplit * kTile)-pixel tile is composited as kSplit^2
// kTile-pixel quadrants (one work item each).
template <int kTile, bool kFull, bool kTrain, int kSplit = 1, int kShape = kShapeDefault>
void launch_composite(const CompositeParams& cp, int64_t max_items, int sms, cudaStream_t stream) {
  const int threads = CompositeGeometry<kTile, CompositeShape<kShape>::kPix>::kThreads;
  max_items *= kSplit * kSplit;
  unsigned grid = static_cast<unsigned>(max_items);
  if (cp.persistent) {
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, composite_kernel<kTile, kFull, kTrain, kSplit, kShape>,
                                                      threads, 0) != cudaSuccess ||
        per_sm < 1) {
      cudaGetLastError();
      per_sm = 1;
    }
    const int64_t resident = static_cast<int64_t>(sms) * per_sm;
    if (resident < max_items) grid = static_cast<unsigned>(resident);
  }
  composite_kernel<kTile, kFull, kTrain, kSplit, kShape><<<grid, threads, 0, stream>>>(cp);
}

// Forward screen-space compositor of one tile size in the requested CTA
// shape (vgr_render_options.composite_shape; 4-pixel tiles have one shape).
template <int kTile, int kSplit = 1>
void launch_forward_composite(const CompositeParams& cp, bool full, int shape, int64_t max_items, int sms,
                              cudaStream_t stream) {
  if (kTile == 4 || shape == kShapeDefault) {
    if (full) launch_composite<kTile, true, false, kSplit>(cp, max_items, sms, stream);
    else launch_composite<kTile, false, false, kSplit>(cp, max_items, sms, stream);
  } else if (shape == kShapeOnePixel) {
    if (full) launch_composite<kTile, true, false, kSplit, kShapeOnePixel>(cp, max_items, sms, stream);
    else launch_composite<kTile, false, false, kSplit, kShapeOnePixel>(cp, max_items, sms, stream);
  } else {
    if (full) launch_composite<kTile, true, false, kSplit, kShapeHalfOccupancy>(cp, max_items, sms, stream);
    else launch_composite<kTile, false, false, kSplit, kShapeHalfOccupancy>(cp, max_items, sms, stream);
  }
}

int render_camera(const vgr_scene* scene, const vgr_cameras* cams, const vgr_outputs* out,
                  const vgr_workspace* ws, const vgr_render_options* opt, void* stream_ptr,
                  int64_t* sorted_buffer_selector, const TrainHooks* train) {
  if (!scene || !cams || !out || !ws || !opt || !sorted_buffer_selector) {
    return fail(VGR_ERR_INVALID_ARGUMENT, "render arguments must be non-null");
  }
  cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
  const bool ragged = cams->widths != nullptr;
  const bool ray = opt->ray_gaussian_evaluation != 0;
  if (!ragged && (opt->height <= 0 || opt->width <= 0)) {
    return fail(VGR_ERR_INVALID_ARGUMENT, "height and width must be positive");
  }
  if (opt->height > INT_MAX || opt->width > INT_MAX) {
    return fail(VGR_ERR_INVALID_ARGUMENT, "resolution exceeds int32 range");
  }
  if (scene->max_scene_gaussians <= 0) {
    return fail(VGR_ERR_INVALID_ARGUMENT, "max_scene_gaussians must be positive");
  }
  if (scene->gaussian_count < 0 || scene->gaussian_count > INT_MAX) {
    return fail(VGR_ERR_INVALID_ARGUMENT, "packed Gaussian ids must fit int32");
  }
  if (scene->max_scene_gaussians > INT_MAX) {
    return fail(VGR_ERR_INVALID_ARGUMENT, "max_scene_gaussians exceeds the first implementation limit");
  }
  if (!(opt->near_plane > 0.0)) return fail(VGR_ERR_INVALID_ARGUMENT, "near_plane must be positive");
  if (!(opt->far_plane > opt->near_plane)) {
    return fail(VGR_ERR_INVALID_ARGUMENT, "far_plane must be greater than near_plane");
  }
  if (!(opt->gaussian_support_sigma > 0.0)) {
    return fail(VGR_ERR_INVALID_ARGUMENT, "gaussian_support_sigma must be positive");
  }
  if (!std::isfinite(opt->covariance_epsilon) || opt->covariance_epsilon < 0.0) {
    return fail(VGR_ERR_INVALID_ARGUMENT, "covariance_epsilon must be finite and non-negative");
  }
  if (!std::isfinite(opt->semantic_min_alpha) || opt->semantic_min_alpha < 0.0 ||
      opt->semantic_min_alpha > 1.0) {
    return fail(VGR_ERR_INVALID_ARGUMENT, "semantic_min_alpha must be finite and in [0, 1]");
  }
  if (opt->composite_shape < kShapeDefault || opt->composite_shape > kShapeHalfOccupancy) {
    return fail(VGR_ERR_INVALID_ARGUMENT, "composite_shape must be 0, 1 or 2");
  }
  const int ts = opt->tile_size;
  if (ts <= 0 || ts > 32 || (ts & (ts - 1)) != 0) {
    return fail(VGR_ERR_INVALID_ARGUMENT, "tile_size must be a power of two in [1, 32]");
  }
  if (ts == 2) {
    return fail(VGR_ERR_UNSUPPORTED, "tile_size=2 is not provided; use 1 (dense mode), 4, 8 or 16");
  }
  if (opt->compact_projection_cache && ts != 1) {
    return fail(VGR_ERR_INVALID_ARGUMENT, "compact_projection_cache requires tile_size=1");
  }
  if (opt->compact_projection_cache && opt->ray_gaussian_evaluation) {
    return fail(VGR_ERR_INVALID_ARGUMENT, "compact_projection_cache supports only screen-space evaluation");
  }
  if (opt->antialiased && opt->ray_gaussian_evaluation) {
    return fail(VGR_ERR_INVALID_ARGUMENT,
                "antialiased rasterization is incompatible with exact-ray evaluation");
  }
  if (opt->sh_degree < -1 || opt->sh_degree > 3) {
    return fail(VGR_ERR_INVALID_ARGUMENT, "sh_degree must be -1 (linear RGB) or in [0, 3]");
  }
  const int64_t min_features =
      opt->sh_degree < 0 ? 3 : static_cast<int64_t>((opt->sh_degree + 1) * (opt->sh_degree + 1) * 3);
  if (scene->feature_width < min_features) {
    return fail(VGR_ERR_INVALID_ARGUMENT,
                opt->sh_degree < 0 ? "features must provide at least RGB channels"
                                   : "features are too narrow for the requested SH degree");
  }
  if (!scene->means || !scene->covariances || !scene->opacities || !scene->features ||
      !scene->semantic_ids || !scene->registered_scene_ids || !scene->scene_offsets) {
    return fail(VGR_ERR_INVALID_ARGUMENT, "scene tensors must be non-null");
  }
  if (!cams->viewmats || !cams->intrinsics || !cams->env_xforms || !cams->camera_scene_ids) {
    return fail(VGR_ERR_INVALID_ARGUMENT, "camera tensors must be non-null");
  }
  if (cams->batch < 0 || cams->batch > INT_MAX) {
    return fail(VGR_ERR_INVALID_ARGUMENT, "camera batch must be in [0, INT_MAX]");
  }
  const int64_t active = cams->active_camera_ids ? cams->active_count : cams->batch;
  if (active < 0 || active > INT_MAX) {
    return fail(VGR_ERR_INVALID_ARGUMENT, "active camera count must be in [0, INT_MAX]");
  }
  if (!out->rgb || (opt->full_sensor_output && (!out->depth || !out->alpha || !out->semantic))) {
    return fail(VGR_ERR_INVALID_ARGUMENT, "output tensors must be non-null");
  }

  // Exact-ray mode bins the plain form's 16-pixel tiles as 32-pixel tiles
  // (renderer_cuda.cu:2670-2676): ray ellipses are wide, so larger bins
  // cut duplicate keys; every pixel still sees the same records in order.
  // The ragged form's tile offsets are the caller's, in tile_size tiles.
  // Dense mode (tile_size 1, the reference's per-pixel path) runs on
  // 16-pixel tiles with the optical-thickness depth cutoff; each pixel sees
  // the same records in the same order, so images equal the plain path's.
  const bool dense = ts == 1;
  if (dense && (ray || ragged || train)) {
    return fail(VGR_ERR_UNSUPPORTED,
                "dense mode (tile_size=1) is provided for the plain screen-space forward render");
  }
  if (dense && !opt->reuse_projection &&
      (!ws->depth_tau || !ws->tile_cutoff || (reinterpret_cast<uintptr_t>(ws->depth_tau) & 15) != 0)) {
    return fail(VGR_ERR_INVALID_ARGUMENT,
                "dense mode needs depth_tau (16-byte aligned) and tile_cutoff workspaces");
  }
  const int bin = dense ? 16 : (ray && ts == 16 && !ragged) ? 32 : ts;
  if (train && bin == 32) {
    return fail(VGR_ERR_UNSUPPORTED, "the differentiable form renders tile_size 4, 8 or 16");
  }
  int64_t tiles_per_image = 0;
  int64_t global_tiles = 0;
  int tiles_x = 0, tiles_y = 0;
  if (ragged) {
    if (!cams->heights || !cams->tile_offsets || !cams->pixel_offsets) {
      return fail(VGR_ERR_INVALID_ARGUMENT,
                  "the ragged form needs widths, heights, tile_offsets and pixel_offsets");
    }
    global_tiles = cams->total_tiles;
    tiles_per_image = 0;
  } else {
    tiles_x = static_cast<int>((opt->width + bin - 1) / bin);
    tiles_y = static_cast<int>((opt->height + bin - 1) / bin);
    tiles_per_image = static_cast<int64_t>(tiles_x) * tiles_y;
    global_tiles = cams->batch * tiles_per_image;
    if (tiles_x > 65535 || tiles_y > 65535) {
      return fail(VGR_ERR_INVALID_ARGUMENT, "at most 65535 tiles per image row or column");
    }
  }
  if (global_tiles > UINT32_MAX) {
    return fail(VGR_ERR_INVALID_ARGUMENT, "global tile count exceeds the uint32 key range");
  }
  if (global_tiles > INT_MAX) {
    return fail(VGR_ERR_INVALID_ARGUMENT, "device tile grouping supports at most INT_MAX tile segments");
  }
  if (ws->tile_capacity < global_tiles) {
    return fail(VGR_ERR_INVALID_ARGUMENT, "tile range workspace is too small for the render batch");
  }
  if (ws->visible_capacity <= 0) return fail(VGR_ERR_INVALID_ARGUMENT, "visible capacity must be positive");
  if (ws->visible_capacity > INT_MAX) {
    return fail(VGR_ERR_INVALID_ARGUMENT, "dense depth ordering requires visible capacity to fit int32");
  }
  if (ws->intersection_capacity <= 0) {
    return fail(VGR_ERR_INVALID_ARGUMENT, "intersection capacity must be positive");
  }
  if (ws->intersection_capacity > INT_MAX) {
    return fail(VGR_ERR_INVALID_ARGUMENT,
                "The first renderer implementation supports at most INT_MAX intersections");
  }
  if (!ws->records || !ws->keys_in || !ws->keys_out || !ws->values_in || !ws->values_out ||
      !ws->tile_starts || !ws->tile_ends || !ws->counters || !ws->scratch) {
    return fail(VGR_ERR_INVALID_ARGUMENT, "workspace tensors must be non-null");
  }
  if ((reinterpret_cast<uintptr_t>(ws->records) & 15) != 0 ||
      (reinterpret_cast<uintptr_t>(ws->scratch) & 255) != 0) {
    return fail(VGR_ERR_INVALID_ARGUMENT,
                "records must be 16-byte aligned and scratch 256-byte aligned");
  }

  const int64_t vblocks = render_vblocks(active, scene->max_scene_gaussians);
  // The 32-bit ticket queue runs past the last virtual block by at most one
  // batch per resident CTA.
  if (vblocks >= static_cast<int64_t>(UINT32_MAX) - (int64_t{1} << 24)) {
    return fail(VGR_ERR_INVALID_ARGUMENT,
                "active cameras x max_scene_gaussians exceeds 2^41 projection tasks");
  }
  const ScratchLayout layout = make_scratch_layout(ws->intersection_capacity, active, false);
  if (ws->scratch_bytes < layout.total) {
    return fail(VGR_ERR_SCRATCH_TOO_SMALL,
                "render scratch holds %lld bytes but this batch needs %lld",
                static_cast<long long>(ws->scratch_bytes), static_cast<long long>(layout.total));
  }

  const float near_f = static_cast<float>(opt->near_plane);
  const float far_f = static_cast<float>(opt->far_plane);

  int sms = 0;
  int rc = device_sms(&sms);
  if (rc != VGR_OK) return rc;

  if (opt->stage_events && opt->stage_event_count != VGR_STAGE_EVENTS) {
    return fail(VGR_ERR_INVALID_ARGUMENT, "stage_events needs exactly %d events", VGR_STAGE_EVENTS);
  }
  auto mark = [&](int i) {
    if (opt->stage_events) cudaEventRecord(static_cast<cudaEvent_t>(opt->stage_events[i]), stream);
  };
  mark(0);
  unsigned char* scratch = static_cast<unsigned char*>(ws->scratch);
  const int32_t* sorted_values = opt->sorted_buffer_hint ? ws->values_out : ws->values_in;
  int64_t selector = 1;

  if (!opt->reuse_projection) {
    if (global_tiles > 0 &&
        cudaMemsetAsync(ws->tile_ends, 0, static_cast<size_t>(global_tiles) * 4, stream) != cudaSuccess) {
      return check_launch("render: clear tile counts", 0);
    }
    SetupParams sp{};
    sp.scratch = scratch;
    sp.layout = layout;
    sp.counters = ws->counters;
    sp.reset_counters = 1;
    sp.active_ids = cams->active_camera_ids;
    sp.active_count = active;
    sp.batch = cams->batch;
    sp.camera_scene_ids = cams->camera_scene_ids;
    sp.registered_scene_ids = scene->registered_scene_ids;
    sp.scene_offsets = scene->scene_offsets;
    sp.scene_count = static_cast<int>(scene->scene_count);
    sp.widths = cams->widths;
    sp.heights = cams->heights;
    sp.tile_offsets = cams->tile_offsets;
    sp.pixel_offsets = cams->pixel_offsets;
    sp.width = static_cast<int>(opt->width);
    sp.height = static_cast<int>(opt->height);
    sp.tile_size = bin;
    sp.viewmats = cams->viewmats;
    sp.intrinsics = cams->intrinsics;
    sp.env_xforms = cams->env_xforms;
    camera_setup_kernel<<<1, 1024, 0, stream>>>(sp);
    if ((rc = check_launch("render: camera setup")) != VGR_OK) return rc;
    mark(1);

    if (train) {
      const int64_t map_elems = active * scene->max_scene_gaussians;
      if (map_elems > 0 &&
          cudaMemsetAsync(train->record_map, 0xff, static_cast<size_t>(map_elems) * 4, stream) !=
              cudaSuccess) {
        return check_launch("render: clear record map", 0);
      }
    }
    ProjectParams pp{};
    pp.scratch = scratch;
    pp.layout = layout;
    pp.means = scene->means;
    pp.covariances = scene->covariances;
    pp.opacities = scene->opacities;
    pp.features = scene->features;
    pp.feature_width = scene->feature_width;
    pp.vector_feature_loads = (reinterpret_cast<uintptr_t>(scene->features) & 15) == 0 &&
                              (scene->feature_width & 3) == 0;
    pp.wide_feature_loads = (reinterpret_cast<uintptr_t>(scene->features) & 31) == 0 &&
                            (scene->feature_width & 7) == 0;
    pp.viewmats = cams->viewmats;
    pp.intrinsics = cams->intrinsics;
    pp.env_xforms = cams->env_xforms;
    pp.active_count = active;
    pp.total_vblocks = vblocks;
    pp.near_plane = near_f;
    pp.far_plane = far_f;
    pp.support_sigma = static_cast<float>(opt->gaussian_support_sigma);
    pp.cov_eps = static_cast<float>(opt->covariance_epsilon);
    pp.antialiased = opt->antialiased != 0;
    pp.tile_size = bin;
    pp.records = ws->records;
    pp.visible_capacity = ws->visible_capacity;
    pp.keys = ws->keys_in;
    pp.values = ws->values_in;
    pp.intersection_capacity = ws->intersection_capacity;
    pp.tile_counts = reinterpret_cast<uint32_t*>(ws->tile_ends);
    pp.tile_count = global_tiles;
    pp.counters = ws->counters;
    pp.mirror_means2d = ws->visible_means2d;
    pp.mirror_conics = ws->visible_conics;
    pp.mirror_depths = ws->visible_depths;
    pp.mirror_opacities = ws->visible_opacities;
    pp.mirror_camera_ids = ws->visible_camera_ids;
    pp.mirror_gaussian_ids = ws->visible_gaussian_ids;
    pp.mirror_radii = ws->visible_radii;
    if (ray && ws->visible_ray_precisions && ws->visible_ray_precision_means) {
      pp.mirror_ray_precisions = ws->visible_ray_precisions;
      pp.mirror_ray_precision_means = ws->visible_ray_precision_means;
    }
    pp.record_map = train ? train->record_map : nullptr;
    pp.record_map_stride = scene->max_scene_gaussians;
    pp.gaussian_ids = scene->gaussian_ids;
    pp.chunk_bounds = reinterpret_cast<const float4*>(scene->chunk_bounds);
    pp.chunk_offsets = scene->chunk_offsets;
    pp.cluster_bounds = scene->chunk_bounds ? reinterpret_cast<const float4*>(scene->cluster_bounds) : nullptr;
    if (scene->chunk_bounds &&
        (!scene->chunk_offsets || (reinterpret_cast<uintptr_t>(scene->chunk_bounds) & 15) != 0)) {
      return fail(VGR_ERR_INVALID_ARGUMENT,
                  "chunk_bounds must be 16-byte aligned and come with chunk_offsets");
    }
    if ((reinterpret_cast<uintptr_t>(scene->cluster_bounds) & 15) != 0) {
      return fail(VGR_ERR_INVALID_ARGUMENT, "cluster_bounds must be 16-byte aligned");
    }
    if (pp.mirror_means2d && !(pp.mirror_conics && pp.mirror_depths && pp.mirror_opacities &&
                               pp.mirror_camera_ids && pp.mirror_gaussian_ids && pp.mirror_radii)) {
      return fail(VGR_ERR_INVALID_ARGUMENT, "the visible-record mirrors must be all set or all null");
    }
    int64_t pgrid = static_cast<int64_t>(sms) * g_occ.project_blocks;
    if (pgrid > vblocks) pgrid = vblocks;
    if (pgrid < 1) pgrid = 1;
    const unsigned pg = static_cast<unsigned>(pgrid);
    if (dense) {
      const int sub_x = static_cast<int>((opt->width + kDenseSubtile - 1) / kDenseSubtile);
      const int sub_y = static_cast<int>((opt->height + kDenseSubtile - 1) / kDenseSubtile);
      const int64_t cells = cams->batch * sub_x * sub_y;
      if (ws->depth_tau_capacity < cells * kDenseBuckets || ws->tile_cutoff_capacity < global_tiles) {
        return fail(VGR_ERR_INVALID_ARGUMENT, "dense-mode workspaces are too small for the pixel grid");
      }
      if (cells > 0 &&
          (cudaMemsetAsync(ws->depth_tau, 0, static_cast<size_t>(cells) * kDenseBuckets * 4, stream) != cudaSuccess ||
           cudaMemsetAsync(ws->tile_cutoff, 0, static_cast<size_t>(global_tiles) * 4, stream) != cudaSuccess)) {
        return check_launch("render: clear depth buckets", 0);
      }
      pp.depth_tau = ws->depth_tau;
      pp.tile_cutoff = ws->tile_cutoff;
      pp.sub_x = sub_x;
      pp.sub_y = sub_y;
      pp.near_bits = [](float f) { uint32_t u; memcpy(&u, &f, 4); return u; }(near_f);
      switch (opt->sh_degree) {
        case -1: project_emit_kernel<-1, false, kProjectDenseTau><<<pg, kProjectThreads, 0, stream>>>(pp); break;
        case 0: project_emit_kernel<0, false, kProjectDenseTau><<<pg, kProjectThreads, 0, stream>>>(pp); break;
        case 1: project_emit_kernel<1, false, kProjectDenseTau><<<pg, kProjectThreads, 0, stream>>>(pp); break;
        case 2: project_emit_kernel<2, false, kProjectDenseTau><<<pg, kProjectThreads, 0, stream>>>(pp); break;
        default: project_emit_kernel<3, false, kProjectDenseTau><<<pg, kProjectThreads, 0, stream>>>(pp); break;
      }
      if ((rc = check_launch("render: dense optical thickness")) != VGR_OK) return rc;
      DenseCutoffParams dp{};
      dp.scratch = scratch;
      dp.layout = layout;
      dp.depth_tau = ws->depth_tau;
      dp.tile_cutoff = ws->tile_cutoff;
      dp.sub_count = cells;
      dp.sub_x = sub_x;
      dp.sub_y = sub_y;
      dp.tiles_x = tiles_x;
      dp.tiles_per_image = tiles_per_image;
      dp.tile_size = bin;
      const int64_t cblocks = (cells * 32 + 255) / 256;
      dense_cutoff_kernel<<<static_cast<unsigned>(cblocks > 0 ? cblocks : 1), 256, 0, stream>>>(dp);
      if ((rc = check_launch("render: dense cutoff")) != VGR_OK) return rc;
      switch (opt->sh_degree) {
        case -1: project_emit_kernel<-1, false, kProjectDenseCull><<<pg, kProjectThreads, 0, stream>>>(pp); break;
        case 0: project_emit_kernel<0, false, kProjectDenseCull><<<pg, kProjectThreads, 0, stream>>>(pp); break;
        case 1: project_emit_kernel<1, false, kProjectDenseCull><<<pg, kProjectThreads, 0, stream>>>(pp); break;
        case 2: project_emit_kernel<2, false, kProjectDenseCull><<<pg, kProjectThreads, 0, stream>>>(pp); break;
        default: project_emit_kernel<3, false, kProjectDenseCull><<<pg, kProjectThreads, 0, stream>>>(pp); break;
      }
    } else if (ray) {
      pp.ray_ext = static_cast<float4*>(ws->records) + ws->visible_capacity * 3;
      switch (opt->sh_degree) {
        case -1: project_emit_kernel<-1, true, kProjectPlain><<<pg, kProjectThreads, 0, stream>>>(pp); break;
        case 0: project_emit_kernel<0, true, kProjectPlain><<<pg, kProjectThreads, 0, stream>>>(pp); break;
        case 1: project_emit_kernel<1, true, kProjectPlain><<<pg, kProjectThreads, 0, stream>>>(pp); break;
        case 2: project_emit_kernel<2, true, kProjectPlain><<<pg, kProjectThreads, 0, stream>>>(pp); break;
        default: project_emit_kernel<3, true, kProjectPlain><<<pg, kProjectThreads, 0, stream>>>(pp); break;
      }
    } else {
      switch (opt->sh_degree) {
        case -1: project_emit_kernel<-1, false, kProjectPlain><<<pg, kProjectThreads, 0, stream>>>(pp); break;
        case 0: project_emit_kernel<0, false, kProjectPlain><<<pg, kProjectThreads, 0, stream>>>(pp); break;
        case 1: project_emit_kernel<1, false, kProjectPlain><<<pg, kProjectThreads, 0, stream>>>(pp); break;
        case 2: project_emit_kernel<2, false, kProjectPlain><<<pg, kProjectThreads, 0, stream>>>(pp); break;
        default: project_emit_kernel<3, false, kProjectPlain><<<pg, kProjectThreads, 0, stream>>>(pp); break;
      }
    }
    if ((rc = check_launch("render: projection")) != VGR_OK) return rc;
    mark(2);

    BucketParams bp{};
    bp.scratch = scratch;
    bp.layout = layout;
    bp.counters = ws->counters;
    bp.capacity = ws->intersection_capacity;
    bp.tile_count = global_tiles;
    bp.keys_in = ws->keys_in;
    bp.values_in = ws->values_in;
    bp.keys_out = ws->keys_out;
    bp.values_out = ws->values_out;
    bp.temp = ws->keys_in;
    bp.tile_starts = ws->tile_starts;
    bp.tile_ends = ws->tile_ends;
    bp.records = static_cast<const Record*>(ws->records);
    bp.visible_capacity = ws->visible_capacity;
    {
      const int64_t spans = (global_tiles + kTileScanSpan - 1) / kTileScanSpan;
      if (spans > 0) {
        tile_span_sum_kernel<<<static_cast<unsigned>(spans), kTileSpanThreads, 0, stream>>>(bp);
        if ((rc = check_launch("render: tile scan (sums)")) != VGR_OK) return rc;
      }
      tile_span_scan_kernel<<<1, kTileScanThreads, 0, stream>>>(bp, spans);
      if ((rc = check_launch("render: tile scan (spans)")) != VGR_OK) return rc;
      if (spans > 0) {
        tile_span_apply_kernel<<<static_cast<unsigned>(spans), kTileSpanThreads, 0, stream>>>(bp);
        if ((rc = check_launch("render: tile scan")) != VGR_OK) return rc;
      }
    }
    mark(3);
    int64_t sgrid = (ws->intersection_capacity + 2047) / 2048;
    // 16 CTAs per SM of grid-stride scatter (8: 1.09 ms, 16: 1.03 ms per
    // 113.6M keys; 4: 1.18 ms).
    if (sgrid > static_cast<int64_t>(sms) * 16) sgrid = static_cast<int64_t>(sms) * 16;
    if (sgrid < 1) sgrid = 1;
    bucket_scatter_kernel<<<static_cast<unsigned>(sgrid), 256, 0, stream>>>(bp);
    if ((rc = check_launch("render: bucket scatter")) != VGR_OK) return rc;
    mark(4);
    bp.large_workers = static_cast<int64_t>(sms) * 4;  // one per resident tile-sort CTA
    bp.large_list = ws->values_in;
    if (global_tiles + bp.large_workers > INT_MAX) {
      return fail(VGR_ERR_INVALID_ARGUMENT, "tile sort grid exceeds CUDA limit");
    }
    large_tile_list_kernel<<<static_cast<unsigned>((global_tiles + 255) / 256), 256, 0, stream>>>(bp);
    if ((rc = check_launch("render: large tile list")) != VGR_OK) return rc;
    tile_sort_kernel<<<static_cast<unsigned>(global_tiles + bp.large_workers), kTileSortThreads, 0, stream>>>(bp);
    if ((rc = check_launch("render: tile sort")) != VGR_OK) return rc;
    selector = 1;
    sorted_values = ws->values_out;
    mark(5);
  }

  for (int i = 1; i <= 5; ++i) {
    if (opt->reuse_projection) mark(i);
  }
  // Compositor over every tile of every active camera.
  const int64_t max_items =
      ragged ? active * cams->max_tiles_per_camera : active * tiles_per_image;
  if (max_items > 0) {
    if (max_items > INT_MAX) return fail(VGR_ERR_INVALID_ARGUMENT, "raster grid exceeds CUDA limit");
    CompositeParams cp{};
    cp.scratch = scratch;
    cp.layout = layout;
    cp.active_count = active;
    cp.tiles_per_camera_hint = ragged ? 0 : tiles_per_image;
    cp.records = static_cast<const Record*>(ws->records);
    cp.values = sorted_values;
    cp.tile_starts = ws->tile_starts;
    cp.tile_ends = ws->tile_ends;
    cp.semantic_ids = scene->semantic_ids;
    cp.semantic_min_alpha = static_cast<float>(opt->semantic_min_alpha);
    cp.output_srgb = opt->output_srgb != 0;
    cp.rgb = out->rgb;
    cp.depth = out->depth;
    cp.alpha = out->alpha;
    cp.semantic = out->semantic;
    cp.final_transmittance = train ? train->final_transmittance : nullptr;
    cp.last_position = train ? train->last_position : nullptr;
    cp.persistent = opt->persistent_compositor != 0;
    const bool full = opt->full_sensor_output != 0;
    if (ray) {
      cp.ray_ext = static_cast<const float4*>(ws->records) + ws->visible_capacity * 3;
      cp.intrinsics = cams->intrinsics;
      cp.support_sigma = static_cast<float>(opt->gaussian_support_sigma);
      const unsigned grid = static_cast<unsigned>(max_items);
      if (bin == 32) {
        if (max_items * 4 > INT_MAX) return fail(VGR_ERR_INVALID_ARGUMENT, "raster grid exceeds CUDA limit");
        const unsigned grid4 = static_cast<unsigned>(max_items * 4);
        if (full) composite_ray_kernel<16, true, 2><<<grid4, composite_threads(16), 0, stream>>>(cp);
        else composite_ray_kernel<16, false, 2><<<grid4, composite_threads(16), 0, stream>>>(cp);
      } else if (bin == 16) {
        if (full) composite_ray_kernel<16, true, 1><<<grid, composite_threads(16), 0, stream>>>(cp);
        else composite_ray_kernel<16, false, 1><<<grid, composite_threads(16), 0, stream>>>(cp);
      } else if (bin == 8) {
        if (full) composite_ray_kernel<8, true, 1><<<grid, composite_threads(8), 0, stream>>>(cp);
        else composite_ray_kernel<8, false, 1><<<grid, composite_threads(8), 0, stream>>>(cp);
      } else {
        if (full) composite_ray_kernel<4, true, 1><<<grid, composite_threads(4), 0, stream>>>(cp);
        else composite_ray_kernel<4, false, 1><<<grid, composite_threads(4), 0, stream>>>(cp);
      }
    } else if (train) {
      if (bin == 16) launch_composite<16, true, true>(cp, max_items, sms, stream);
      else if (bin == 8) launch_composite<8, true, true>(cp, max_items, sms, stream);
      else launch_composite<4, true, true>(cp, max_items, sms, stream);
    } else if (bin == 32) {
      if (max_items * 4 > INT_MAX) return fail(VGR_ERR_INVALID_ARGUMENT, "raster grid exceeds CUDA limit");
      launch_forward_composite<16, 2>(cp, full, opt->composite_shape, max_items, sms, stream);
    } else if (bin == 16) {
      launch_forward_composite<16>(cp, full, opt->composite_shape, max_items, sms, stream);
    } else if (bin == 8) {
      launch_forward_composite<8>(cp, full, opt->composite_shape, max_items, sms, stream);
    } else {
      launch_forward_composite<4>(cp, full, opt->composite_shape, max_items, sms, stream);
    }
    if ((rc = check_launch("render: compositor")) != VGR_OK) return rc;
  }
  mark(6);
  *sorted_buffer_selector = selector;
  return VGR_OK;
}

}  // namespace vgr

extern "C" int vgr_render(const vgr_scene* scene, const vgr_cameras* cams,
                          const vgr_outputs* out, const vgr_workspace* ws,
                          const vgr_render_options* opt, void* stream_ptr,
                          int64_t* sorted_buffer_selector) {
  return vgr::render_camera(scene, cams, out, ws, opt, stream_ptr, sorted_buffer_selector, nullptr);
}
