// Depth-ordered straight-alpha composite of a Gaussian layer and a mesh layer
// (src/isaacsim_gaussian_renderer/hybrid_compositor.py:21-128), one thread per
// pixel instead of the reference's chain of ~20 elementwise tensor passes.
// Every operation is an explicit round-to-nearest intrinsic in the
// reference's evaluation order, so the result equals the reference's float32
// tensor expression bit for bit.
#include <cuda_runtime.h>

#include <climits>
#include <cmath>

#include "../../include/vgr_b200.h"
#include "vgr_api_internal.h"
#include "vgr_common.cuh"

namespace vgr {
namespace {

struct HybridParams {
  const float* g_rgb;
  const float* g_alpha;
  const float* g_depth;
  const float* m_rgb;
  const float* m_alpha;
  const float* m_depth;
  int64_t pixels;
  float min_alpha;
  float depth_epsilon;
  float* rgb;
  float* alpha;
  float* depth;
  uint8_t* mesh_in_front;
};

__global__ void __launch_bounds__(256) hybrid_composite_kernel(HybridParams p) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= p.pixels) return;
  const float ga = p.g_alpha[i], gd = p.g_depth[i];
  const float ma = p.m_alpha[i], md = p.m_depth[i];
  const bool gv = ga > p.min_alpha && isfinite(ga) && isfinite(gd);
  const bool mv = ma > p.min_alpha && isfinite(ma) && isfinite(md);
  const bool front_mesh = mv && (!gv || fadd(md, p.depth_epsilon) < gd);
  const float ga_v = gv ? ga : 0.0f;
  const float ma_v = mv ? ma : 0.0f;
  const float front_a = front_mesh ? ma_v : ga_v;
  const float back_a = front_mesh ? ga_v : ma_v;
  const float keep = fsub(1.0f, front_a);
  const float out_alpha = fadd(front_a, fmul(back_a, keep));
  const float eps = 1.1920928955078125e-07f;  // float32 machine epsilon
  const float denom = fmaxf(out_alpha, eps);
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const float g = gv ? p.g_rgb[i * 3 + c] : 0.0f;
    const float m = mv ? p.m_rgb[i * 3 + c] : 0.0f;
    const float front = front_mesh ? m : g;
    const float back = front_mesh ? g : m;
    const float prem = fadd(fmul(front, front_a), fmul(fmul(back, back_a), keep));
    p.rgb[i * 3 + c] = out_alpha > p.min_alpha ? fdiv(prem, denom) : 0.0f;
  }
  p.alpha[i] = out_alpha;
  p.depth[i] = (gv || mv) ? (front_mesh ? md : gd) : __int_as_float(0x7f800000);
  p.mesh_in_front[i] = front_mesh ? 1 : 0;
}

}  // namespace
}  // namespace vgr

extern "C" int vgr_composite_gaussian_and_mesh(
    const float* gaussian_rgb, const float* gaussian_alpha, const float* gaussian_depth,
    const float* mesh_rgb, const float* mesh_alpha, const float* mesh_depth, int64_t pixels,
    double min_alpha, double depth_epsilon, float* rgb, float* alpha, float* depth,
    uint8_t* mesh_in_front, void* stream) {
  if (!gaussian_rgb || !gaussian_alpha || !gaussian_depth || !mesh_rgb || !mesh_alpha ||
      !mesh_depth || !rgb || !alpha || !depth || !mesh_in_front) {
    return vgr::fail(VGR_ERR_INVALID_ARGUMENT, "hybrid composite arguments must be non-null");
  }
  if (!(min_alpha >= 0.0 && min_alpha <= 1.0)) {
    return vgr::fail(VGR_ERR_INVALID_ARGUMENT, "min_alpha must be in [0, 1].");
  }
  if (!(depth_epsilon >= 0.0)) {
    return vgr::fail(VGR_ERR_INVALID_ARGUMENT, "depth_epsilon must be non-negative.");
  }
  if (pixels < 0) return vgr::fail(VGR_ERR_INVALID_ARGUMENT, "pixels must be non-negative");
  if (pixels == 0) return VGR_OK;
  const int64_t blocks = (pixels + 255) / 256;
  if (blocks > INT_MAX) return vgr::fail(VGR_ERR_INVALID_ARGUMENT, "pixel count exceeds the grid limit");
  vgr::HybridParams p{gaussian_rgb, gaussian_alpha, gaussian_depth, mesh_rgb, mesh_alpha, mesh_depth,
                      pixels, static_cast<float>(min_alpha), static_cast<float>(depth_epsilon),
                      rgb, alpha, depth, mesh_in_front};
  vgr::hybrid_composite_kernel<<<static_cast<unsigned>(blocks), 256, 0,
                                 static_cast<cudaStream_t>(stream)>>>(p);
  return vgr::check_launch("hybrid composite");
}
