// Helpers shared by the C ABI translation units.
#pragma once

#include <stdint.h>

#include "../../include/vgr_b200.h"

namespace vgr {

// Records a thread-local error message and returns code.
int fail(int code, const char* fmt, ...);
// Converts a pending CUDA launch error into VGR_ERR_CUDA.
int check_launch(const char* what, int launches = 1);
// Streaming-multiprocessor count of the current device (cached).
int device_sms(int* sms);

// Training outputs of the camera forward (all non-null when training).
struct TrainHooks {
  float* final_transmittance;  // [P]
  int32_t* last_position;      // [P]
  int32_t* record_map;         // [A, max_scene_gaussians]
};

// vgr_render with optional training outputs.
int render_camera(const vgr_scene* scene, const vgr_cameras* cams, const vgr_outputs* out,
                  const vgr_workspace* ws, const vgr_render_options* opt, void* stream,
                  int64_t* sorted_buffer_selector, const TrainHooks* train);

}  // namespace vgr
