// C ABI of the differentiable camera form (declared in include/vgr_b200.h).
//
// vgr_render_train is vgr_render with the training outputs switched on (the
// record map written by the projection, final transmittance and last blended
// position per pixel written by the compositor); vgr_render_backward runs the
// compositor backward and the per-Gaussian projection backward on the same
// stream, reading the forward's scratch (camera plans and projection
// constants), sorted lists and records, which must be untouched since.
#include <cuda_runtime.h>

#include <climits>
#include <cmath>

#include "../../include/vgr_b200.h"
#include "vgr_api_internal.h"
#include "vgr_kernels.h"

using vgr::fail;

namespace {

int check_train_options(const vgr_render_options* opt) {
  if (!opt->full_sensor_output) {
    return fail(VGR_ERR_INVALID_ARGUMENT, "the differentiable form needs full_sensor_output=1");
  }
  if (opt->output_srgb) {
    return fail(VGR_ERR_UNSUPPORTED, "the differentiable form renders linear RGB (output_srgb=0)");
  }
  if (opt->antialiased) {
    return fail(VGR_ERR_UNSUPPORTED, "the differentiable form does not provide antialiased=1");
  }
  if (opt->ray_gaussian_evaluation) {
    return fail(VGR_ERR_UNSUPPORTED, "the differentiable form does not provide ray_gaussian_evaluation=1");
  }
  if (opt->reuse_projection) {
    return fail(VGR_ERR_INVALID_ARGUMENT, "the differentiable form projects every frame");
  }
  return VGR_OK;
}

int check_state(const vgr_scene* scene, const vgr_cameras* cams, const vgr_workspace* ws,
                const vgr_train_state* state) {
  if (!state || !state->final_transmittance || !state->last_position || !state->record_map ||
      !state->record_grads) {
    return fail(VGR_ERR_INVALID_ARGUMENT, "training state buffers must be non-null");
  }
  if ((reinterpret_cast<uintptr_t>(state->record_grads) & 15) != 0) {
    return fail(VGR_ERR_INVALID_ARGUMENT, "record_grads must be 16-byte aligned");
  }
  const int64_t active = cams->active_camera_ids ? cams->active_count : cams->batch;
  if (state->record_map_capacity < active * scene->max_scene_gaussians) {
    return fail(VGR_ERR_INVALID_ARGUMENT,
                "record_map holds %lld elements but the batch needs active cameras x "
                "max_scene_gaussians = %lld",
                static_cast<long long>(state->record_map_capacity),
                static_cast<long long>(active * scene->max_scene_gaussians));
  }
  if (ws->visible_capacity <= 0) {
    return fail(VGR_ERR_INVALID_ARGUMENT, "visible capacity must be positive");
  }
  return VGR_OK;
}

}  // namespace

extern "C" int vgr_train_activate(const vgr_train_params* params, int64_t count,
                                  float* covariances, float* opacities, void* stream) {
  if (!params || !params->log_scales || !params->rotations || !params->opacity_logits ||
      !covariances || !opacities) {
    return fail(VGR_ERR_INVALID_ARGUMENT, "activation arguments must be non-null");
  }
  if (count < 0) return fail(VGR_ERR_INVALID_ARGUMENT, "gaussian_count must be non-negative");
  if (count == 0) return VGR_OK;
  vgr::TrainActivateParams p{};
  p.log_scales = params->log_scales;
  p.rotations = params->rotations;
  p.opacity_logits = params->opacity_logits;
  p.count = count;
  p.covariances = covariances;
  p.opacities = opacities;
  const int64_t blocks = (count + 255) / 256;
  if (blocks > INT_MAX) return fail(VGR_ERR_INVALID_ARGUMENT, "gaussian_count exceeds the grid limit");
  vgr::train_activate_kernel<<<static_cast<unsigned>(blocks), 256, 0,
                               static_cast<cudaStream_t>(stream)>>>(p);
  return vgr::check_launch("train_activate");
}

extern "C" int vgr_render_train(const vgr_scene* scene, const vgr_cameras* cams,
                                const vgr_outputs* out, const vgr_workspace* ws,
                                const vgr_render_options* opt, const vgr_train_state* state,
                                void* stream, int64_t* sorted_buffer_selector) {
  if (!scene || !cams || !out || !ws || !opt) {
    return fail(VGR_ERR_INVALID_ARGUMENT, "render arguments must be non-null");
  }
  int rc = check_train_options(opt);
  if (rc != VGR_OK) return rc;
  rc = check_state(scene, cams, ws, state);
  if (rc != VGR_OK) return rc;
  vgr::TrainHooks hooks{state->final_transmittance, state->last_position, state->record_map};
  return vgr::render_camera(scene, cams, out, ws, opt, stream, sorted_buffer_selector, &hooks);
}

extern "C" int vgr_render_backward(const vgr_scene* scene, const vgr_train_params* params,
                                   const vgr_cameras* cams, const vgr_outputs* out,
                                   const vgr_workspace* ws, const vgr_render_options* opt,
                                   const vgr_train_state* state, const vgr_output_grads* grads,
                                   const vgr_param_grads* pg, void* stream_ptr) {
  if (!scene || !params || !cams || !out || !ws || !opt || !grads || !pg) {
    return fail(VGR_ERR_INVALID_ARGUMENT, "backward arguments must be non-null");
  }
  int rc = check_train_options(opt);
  if (rc != VGR_OK) return rc;
  rc = check_state(scene, cams, ws, state);
  if (rc != VGR_OK) return rc;
  if (!grads->rgb) return fail(VGR_ERR_INVALID_ARGUMENT, "the RGB output gradient must be non-null");
  if (!out->depth) return fail(VGR_ERR_INVALID_ARGUMENT, "the forward depth output must be non-null");
  if (!pg->means || !pg->log_scales || !pg->rotations || !pg->opacity_logits || !pg->features) {
    return fail(VGR_ERR_INVALID_ARGUMENT, "parameter gradient buffers must be non-null");
  }
  if (!params->log_scales || !params->rotations || !params->opacity_logits) {
    return fail(VGR_ERR_INVALID_ARGUMENT, "training parameters must be non-null");
  }
  if (opt->sh_degree < -1 || opt->sh_degree > 3) {
    return fail(VGR_ERR_INVALID_ARGUMENT, "sh_degree must be -1 (linear RGB) or in [0, 3]");
  }
  const int ts = opt->tile_size;
  if (ts != 4 && ts != 8 && ts != 16) {
    return fail(VGR_ERR_INVALID_ARGUMENT, "tile_size must be 4, 8 or 16");
  }
  if (scene->gaussian_count < 0 || scene->gaussian_count > INT_MAX) {
    return fail(VGR_ERR_INVALID_ARGUMENT, "packed Gaussian ids must fit int32");
  }
  cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
  const bool ragged = cams->widths != nullptr;
  const int64_t active = cams->active_camera_ids ? cams->active_count : cams->batch;
  const vgr::ScratchLayout layout = vgr::make_scratch_layout(ws->intersection_capacity, active, false);
  if (ws->scratch_bytes < layout.total || !ws->scratch) {
    return fail(VGR_ERR_SCRATCH_TOO_SMALL, "backward needs the forward's render scratch");
  }
  const unsigned char* scratch = static_cast<const unsigned char*>(ws->scratch);
  float4* record_grads = static_cast<float4*>(state->record_grads);
  int sms = 0;
  rc = vgr::device_sms(&sms);
  if (rc != VGR_OK) return rc;

  vgr::zero_record_grads_kernel<<<static_cast<unsigned>(sms) * 4, 256, 0, stream>>>(
      record_grads, ws->counters, ws->visible_capacity);
  if ((rc = vgr::check_launch("backward: clear record gradients")) != VGR_OK) return rc;

  int64_t tiles_per_image = 0;
  int64_t max_items = 0;
  if (ragged) {
    max_items = active * cams->max_tiles_per_camera;
  } else {
    const int64_t tx = (opt->width + ts - 1) / ts;
    const int64_t ty = (opt->height + ts - 1) / ts;
    tiles_per_image = tx * ty;
    max_items = active * tiles_per_image;
  }
  if (max_items > INT_MAX) return fail(VGR_ERR_INVALID_ARGUMENT, "raster grid exceeds CUDA limit");
  if (max_items > 0) {
    vgr::CompositeBackwardParams cb{};
    cb.scratch = scratch;
    cb.layout = layout;
    cb.active_count = active;
    cb.tiles_per_camera_hint = ragged ? 0 : tiles_per_image;
    cb.records = static_cast<const vgr::Record*>(ws->records);
    cb.values = ws->values_out;
    cb.tile_starts = ws->tile_starts;
    cb.tile_ends = ws->tile_ends;
    cb.final_transmittance = state->final_transmittance;
    cb.last_position = state->last_position;
    cb.depth = out->depth;
    cb.grad_rgb = grads->rgb;
    cb.grad_depth = grads->depth;
    cb.grad_alpha = grads->alpha;
    cb.record_grads = record_grads;
    const unsigned grid = static_cast<unsigned>(max_items);
    if (ts == 16) {
      vgr::composite_backward_kernel<16><<<grid, vgr::composite_threads(16), 0, stream>>>(cb);
    } else if (ts == 8) {
      vgr::composite_backward_kernel<8><<<grid, vgr::composite_threads(8), 0, stream>>>(cb);
    } else {
      vgr::composite_backward_kernel<4><<<grid, vgr::composite_threads(4), 0, stream>>>(cb);
    }
    if ((rc = vgr::check_launch("backward: compositor")) != VGR_OK) return rc;
  }

  const int64_t count = scene->gaussian_count;
  if (count > 0) {
    vgr::ProjectBackwardParams pb{};
    pb.scratch = scratch;
    pb.layout = layout;
    pb.active_count = active;
    pb.scene_offsets = scene->scene_offsets;
    pb.scene_count = static_cast<int>(scene->scene_count);
    pb.gaussian_count = count;
    pb.means = scene->means;
    pb.covariances = scene->covariances;
    pb.opacities = scene->opacities;
    pb.features = scene->features;
    pb.feature_width = scene->feature_width;
    pb.vector_feature_loads = (reinterpret_cast<uintptr_t>(scene->features) & 15) == 0 &&
                              (scene->feature_width & 3) == 0;
    pb.log_scales = params->log_scales;
    pb.rotations = params->rotations;
    pb.cov_eps = static_cast<float>(opt->covariance_epsilon);
    pb.record_map = state->record_map;
    pb.record_map_stride = scene->max_scene_gaussians;
    pb.record_grads = record_grads;
    pb.d_means = pg->means;
    pb.d_log_scales = pg->log_scales;
    pb.d_rotations = pg->rotations;
    pb.d_opacity_logits = pg->opacity_logits;
    pb.d_features = pg->features;
    constexpr int kThreads = 128;  // kProjectBackwardThreads
    const unsigned grid = static_cast<unsigned>((count + kThreads - 1) / kThreads);
    switch (opt->sh_degree) {
      case -1: vgr::project_backward_kernel<-1><<<grid, kThreads, 0, stream>>>(pb); break;
      case 0: vgr::project_backward_kernel<0><<<grid, kThreads, 0, stream>>>(pb); break;
      case 1: vgr::project_backward_kernel<1><<<grid, kThreads, 0, stream>>>(pb); break;
      case 2: vgr::project_backward_kernel<2><<<grid, kThreads, 0, stream>>>(pb); break;
      default: vgr::project_backward_kernel<3><<<grid, kThreads, 0, stream>>>(pb); break;
    }
    if ((rc = vgr::check_launch("backward: projection")) != VGR_OK) return rc;
  }
  return VGR_OK;
}

extern "C" int vgr_photometric_loss(const float* rgb, const float* target_rgb, const float* depth,
                                    const float* target_depth, int64_t pixels, double depth_weight,
                                    float* loss, float* grad_rgb, float* grad_depth,
                                    void* stream_ptr) {
  if (!rgb || !target_rgb || !depth || !target_depth || !loss || !grad_rgb || !grad_depth) {
    return fail(VGR_ERR_INVALID_ARGUMENT, "loss arguments must be non-null");
  }
  if (pixels <= 0) return fail(VGR_ERR_INVALID_ARGUMENT, "pixels must be positive");
  if (!std::isfinite(depth_weight)) return fail(VGR_ERR_INVALID_ARGUMENT, "depth_weight must be finite");
  cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
  if (cudaMemsetAsync(loss, 0, sizeof(float), stream) != cudaSuccess) {
    return vgr::check_launch("photometric loss: clear", 0);
  }
  int sms = 0;
  int rc = vgr::device_sms(&sms);
  if (rc != VGR_OK) return rc;
  vgr::PhotometricLossParams p{};
  p.rgb = rgb;
  p.target_rgb = target_rgb;
  p.depth = depth;
  p.target_depth = target_depth;
  p.pixels = pixels;
  p.depth_weight = static_cast<float>(depth_weight);
  p.loss = loss;
  p.grad_rgb = grad_rgb;
  p.grad_depth = grad_depth;
  int64_t blocks = (pixels + 255) / 256;
  if (blocks > static_cast<int64_t>(sms) * 8) blocks = static_cast<int64_t>(sms) * 8;
  vgr::photometric_loss_kernel<<<static_cast<unsigned>(blocks), 256, 0, stream>>>(p);
  return vgr::check_launch("photometric loss");
}
