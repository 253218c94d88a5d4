// Differentiable camera form: parameter activation, compositor backward and
// per-Gaussian projection backward.
//
// The forward equation is the compositor of
// src/isaacsim_gaussian_renderer/native/renderer_cuda.cu:1973-2305 over the
// projection of :287-490 (the same kernels as the plain form, with the
// training outputs switched on).  The reference renders forward only; its
// gradient baseline is gsplat, whose backward is not available here, so the
// derivatives below are written from the forward equation and checked against
// float64 automatic differentiation and central finite differences.
//
// Forward, per pixel, records i in sorted order:
//   w_i = alpha_i T_i,  T_{i+1} = T_i (1 - alpha_i),  C = sum w_i c_i,
//   A = 1 - T_final,  D = (sum w_i z_i) / A,
//   alpha_i = min(0.99, o_i exp(power_i)),
//   power_i = -(c0 dx^2 + 2 c1 dx dy + c2 dy^2) / 2,  dx = px - mean_x.
// Backward, visiting a pixel's blended records from the last one back:
//   f_i = gC . c_i + gZ z_i  with gZ = gD / A,
//   dL/dalpha_i = f_i T_i + (gA' T_final - S_i) / (1 - alpha_i),
//   S_i = sum_{j > i} f_j w_j,  gA' = gA - gD D / A,
// and T_i = T_{i+1} / (1 - alpha_i) recovers the transmittance.
//
// B200 structure: the compositor backward keeps the forward's CTA shape (two
// pixels per thread, 8x8-pixel warp blocks, the same staged records and warp
// masks, so every alpha decision is the forward's), walks each batch of 256
// records back to front, reduces each record's ten partial derivatives over
// the warp with shuffles into shared memory, and flushes one batch with three
// float4 atomics per touched record.  The projection backward runs one thread
// per Gaussian over every camera that saw it (a (slot, Gaussian) -> record map
// written by the training forward), so the per-Gaussian sums need no atomics,
// and applies the activation derivatives (exp scales, normalised quaternion,
// sigmoid opacity) in the same pass.
#include "vgr_kernels.h"

namespace vgr {

// ---------------------------------------------------------------------------
// Activation: covariance from (log scales, quaternion), opacity = sigmoid.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float clamp_exp_arg(float v) { return fminf(fmaxf(v, -80.0f), 80.0f); }

__global__ void __launch_bounds__(256) train_activate_kernel(TrainActivateParams p) {
  const int64_t g = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (g >= p.count) return;
  float cov[6];
  covariance_from_quaternion(p.rotations[g * 4 + 0], p.rotations[g * 4 + 1], p.rotations[g * 4 + 2],
                             p.rotations[g * 4 + 3], vexp(clamp_exp_arg(p.log_scales[g * 3 + 0])),
                             vexp(clamp_exp_arg(p.log_scales[g * 3 + 1])),
                             vexp(clamp_exp_arg(p.log_scales[g * 3 + 2])), cov);
#pragma unroll
  for (int k = 0; k < 6; ++k) p.covariances[g * 6 + k] = cov[k];
  p.opacities[g] = fdiv(1.0f, fadd(1.0f, vexp(clamp_exp_arg(-p.opacity_logits[g]))));
}

// Clears the record gradients of the frame's visible records (count from the
// device counters, so no host round trip).
__global__ void __launch_bounds__(256) zero_record_grads_kernel(float4* __restrict__ grads,
                                                                const int64_t* __restrict__ counters,
                                                                int64_t capacity) {
  int64_t n = counters[0];
  if (n > capacity) n = capacity;
  const float4 z = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n * 3;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    grads[i] = z;
  }
}

// ---------------------------------------------------------------------------
// Photometric loss L = mean((rgb - t)^2) + w mean(|depth - t_depth|) over the
// pixels where both depths are finite, with its gradient, in one pass.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) photometric_loss_kernel(PhotometricLossParams p) {
  __shared__ float s_warp[8];
  const float rgb_scale = 1.0f / static_cast<float>(3 * p.pixels);
  const float depth_scale = p.depth_weight / static_cast<float>(p.pixels);
  float sum = 0.0f;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < p.pixels;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const float d = p.rgb[i * 3 + c] - p.target_rgb[i * 3 + c];
      sum = fmaf(d * d, rgb_scale, sum);
      p.grad_rgb[i * 3 + c] = 2.0f * rgb_scale * d;
    }
    const float z = p.depth[i];
    const float tz = p.target_depth[i];
    float gz = 0.0f;
    if (isfinite(z) && isfinite(tz)) {
      const float d = z - tz;
      sum = fmaf(fabsf(d), depth_scale, sum);
      gz = d > 0.0f ? depth_scale : (d < 0.0f ? -depth_scale : 0.0f);
    }
    p.grad_depth[i] = gz;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
  if ((threadIdx.x & 31) == 0) s_warp[threadIdx.x >> 5] = sum;
  __syncthreads();
  if (threadIdx.x == 0) {
    float block = 0.0f;
#pragma unroll
    for (int w = 0; w < 8; ++w) block += s_warp[w];
    atomicAdd(p.loss, block);
  }
}

// ---------------------------------------------------------------------------
// Compositor backward.
// ---------------------------------------------------------------------------
// Per-record sums gathered over a record's pixels, in this order: the
// moments of dp = dL/dpower against the pixel offset (dx, dy) from the mean
// (dp dx, dp dy, dp dx^2, dp dx dy, dp dy^2), from which the flush forms the
// mean and conic derivatives with the record's conic; dL/dopacity; the
// colour and depth derivatives.
enum RecordGrad { kMDx, kMDy, kMDxx, kMDxy, kMDyy, kGOpacity, kGRed, kGGreen, kGBlue, kGDepth,
                  kRecordGradCount };
// Shared-memory stride of one record's terms: odd, so that both the lanes
// of a transposed sum (one term each) and the flush (one record each) hit
// distinct banks.
constexpr int kGradStride = kRecordGradCount + 1;

struct PixelGrad {
  float t;       // transmittance after the records not yet visited
  float s;       // sum of f_j w_j over the visited records
  float k;       // gA' * T_final
  float gr, gg, gb, gz;
  int32_t last;  // sorted position one past the last blended record
};

__device__ __forceinline__ PixelGrad load_pixel_grad(const CompositeBackwardParams& p,
                                                     const CamPlan& plan, int x, int y,
                                                     bool valid) {
  PixelGrad q{1.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0};
  if (!valid) return q;
  const int64_t pixel = plan.pixel_base + static_cast<int64_t>(y) * plan.width + x;
  const float tf = p.final_transmittance[pixel];
  q.t = tf;
  q.last = p.last_position[pixel];
  q.gr = p.grad_rgb[pixel * 3 + 0];
  q.gg = p.grad_rgb[pixel * 3 + 1];
  q.gb = p.grad_rgb[pixel * 3 + 2];
  const float ga = p.grad_alpha ? p.grad_alpha[pixel] : 0.0f;
  const float gd = p.grad_depth ? p.grad_depth[pixel] : 0.0f;
  const float a = fsub(1.0f, tf);
  float ga2 = ga;
  if (a > 1.0e-8f && gd != 0.0f) {
    const float d = p.depth[pixel];
    q.gz = gd / a;
    ga2 = ga - gd * d / a;
  }
  q.k = ga2 * tf;
  return q;
}

__device__ __forceinline__ float fast_exp(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x * 1.4426950408889634f));
  return y;
}

__device__ __forceinline__ float fast_rcp(float x) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// One record on one pixel, back to front, without branches: c says whether
// the record was blended into the pixel (power in range, before the pixel's
// last blended record, alpha >= 1/255 on the forward's exact arithmetic).
// A record that was not blended enters with alpha = 0, which leaves the
// pixel state unchanged and adds nothing.  Derivative values use the
// special-function unit's exp and reciprocal (relative error ~1e-7).
// Returns dL/dpower; the caller forms the moments of the thread's pixels
// (which share dx) together.
__device__ __forceinline__ float backward_pixel(PixelGrad& q, bool c, float oe, float e,
                                                const float4& col, float* g) {
  const bool unclamped = c && oe < kMaxAlpha;
  const float alpha = c ? fminf(kMaxAlpha, oe) : 0.0f;
  const float de = unclamped ? e : 0.0f;          // d alpha / d opacity
  const float dpow = unclamped ? alpha : 0.0f;    // d alpha / d power
  const float inv = c ? fast_rcp(1.0f - alpha) : 1.0f;
  const float t_before = q.t * inv;
  const float w = alpha * t_before;
  const float f = q.gr * col.x + q.gg * col.y + q.gb * col.z + q.gz * col.w;
  const float d_alpha = f * t_before + (q.k - q.s) * inv;
  q.s = fmaf(f, w, q.s);
  q.t = t_before;
  g[kGRed] = fmaf(q.gr, w, g[kGRed]);
  g[kGGreen] = fmaf(q.gg, w, g[kGGreen]);
  g[kGBlue] = fmaf(q.gb, w, g[kGBlue]);
  g[kGDepth] = fmaf(q.gz, w, g[kGDepth]);
  g[kGOpacity] = fmaf(d_alpha, de, g[kGOpacity]);
  return d_alpha * dpow;
}

template <int kTile>
__global__ void __launch_bounds__(CompositeGeometry<kTile>::kThreads)
    composite_backward_kernel(CompositeBackwardParams p) {
  using Geo = CompositeGeometry<kTile>;
  __shared__ float4 s_geo[kCompositeBatch];
  __shared__ float4 s_cpo[kCompositeBatch];
  __shared__ float4 s_col[kCompositeBatch];
  __shared__ uint32_t s_mask[kCompositeBatch];
  __shared__ float s_grad[kCompositeBatch * kGradStride];
  __shared__ int32_t s_last[Geo::kWarps];

  CamPlan plan;
  int64_t local_tile;
  if (!locate_tile(p.scratch, p.layout, p.active_count, p.tiles_per_camera_hint, blockIdx.x, plan,
                   local_tile)) {
    return;
  }
  const int tile_y = static_cast<int>(local_tile / plan.tiles_x);
  const int tile_x = static_cast<int>(local_tile - static_cast<int64_t>(tile_y) * plan.tiles_x);
  const int64_t global_tile = plan.tile_base + local_tile;
  const int64_t range_start = p.tile_starts[global_tile];
  const int64_t range_end = p.tile_ends[global_tile];
  if (!(range_start >= 0 && range_end > range_start)) return;

  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  const int lx = lane % Geo::kBlockW;
  const int ly = lane / Geo::kBlockW;
  const bool lane_used = ly < Geo::kLaneRows;
  const int pixel_x = tile_x * kTile + (warp % Geo::kWarpsX) * Geo::kBlockW + lx;
  const int pixel_y0 = tile_y * kTile + (warp / Geo::kWarpsX) * Geo::kBlockH + ly;
  const int pixel_y1 = pixel_y0 + Geo::kLaneRows;
  const bool valid0 = lane_used && pixel_x < plan.width && pixel_y0 < plan.height;
  const bool valid1 = lane_used && pixel_x < plan.width && pixel_y1 < plan.height;
  const float cx = fadd(static_cast<float>(pixel_x), 0.5f);
  const float cy0 = fadd(static_cast<float>(pixel_y0), 0.5f);
  const float cy1 = fadd(static_cast<float>(pixel_y1), 0.5f);
  PixelGrad q0 = load_pixel_grad(p, plan, pixel_x, pixel_y0, valid0);
  PixelGrad q1 = load_pixel_grad(p, plan, pixel_x, pixel_y1, valid1);

  const int32_t warp_last = __reduce_max_sync(0xffffffffu, max(q0.last, q1.last));
  if (lane == 0) s_last[warp] = warp_last;
  __syncthreads();
  int32_t cta_last = 0;
#pragma unroll
  for (int w = 0; w < Geo::kWarps; ++w) cta_last = max(cta_last, s_last[w]);
  const int64_t end = min(range_end, static_cast<int64_t>(cta_last));
  const float tile_x0 = static_cast<float>(tile_x * kTile);
  const float tile_y0 = static_cast<float>(tile_y * kTile);

  for (int64_t hi = end; hi > range_start; hi -= kCompositeBatch) {
    const int64_t lo = max(range_start, hi - kCompositeBatch);
    const int n = static_cast<int>(hi - lo);
    for (int j = tid; j < n; j += Geo::kThreads) {
      stage_composite_record<kTile>(p.records[p.values[lo + j]], tile_x0, tile_y0, s_geo[j],
                                    s_cpo[j], s_col[j], s_mask[j]);
#pragma unroll
      for (int f = 0; f < kRecordGradCount; ++f) s_grad[j * kGradStride + f] = 0.0f;
    }
    __syncthreads();
    if (lo < warp_last) {
      for (int base = (n - 1) & ~31; base >= 0; base -= 32) {
        const uint32_t m = (base + lane < n) ? s_mask[base + lane] : 0u;
        uint32_t bits = __ballot_sync(0xffffffffu, (m >> warp) & 1u);
        while (bits) {
          const int hb = 31 - __clz(bits);
          bits &= ~(1u << hb);
          const int j = base + hb;
          const int32_t pos = static_cast<int32_t>(lo + j);
          if (pos >= warp_last) continue;
          const float4 geo = s_geo[j];
          const float4 cpo = s_cpo[j];
          const float dx = fsub(cx, geo.x);
          const float adx = fmul(fmul(geo.z, dx), dx);
          const float bdx = fmul(geo.w, dx);
          const float dy0 = fsub(cy0, geo.y);
          const float dy1 = fsub(cy1, geo.y);
          const float p0 = ffma(fmul(cpo.x, dy0), dy0, ffma(bdx, dy0, adx));
          const float p1 = ffma(fmul(cpo.x, dy1), dy1, ffma(bdx, dy1, adx));
          const bool in0 = p0 >= cpo.y && p0 <= 0.0f && pos < q0.last;
          const bool in1 = p1 >= cpo.y && p1 <= 0.0f && pos < q1.last;
          // One vote (the ballot below) decides whether the warp takes the
          // record: a vote on in0 || in1 before the two exponentials cost
          // more than the exponentials it skipped.
          const float o = cpo.z;
          float e0 = fast_exp(p0);
          float e1 = fast_exp(p1);
          float oe0 = o * e0;
          float oe1 = o * e1;
          // The 1/255 decision must be the forward's: near it, take it on
          // the forward's exact exp (rare, so warp-uniform).
          const bool near = (in0 && fabsf(oe0 - kAlphaThreshold) <= 1.0e-5f * kAlphaThreshold) ||
                            (in1 && fabsf(oe1 - kAlphaThreshold) <= 1.0e-5f * kAlphaThreshold);
          if (__any_sync(0xffffffffu, near)) {
            e0 = vexp(p0);
            e1 = vexp(p1);
            oe0 = fmul(o, e0);
            oe1 = fmul(o, e1);
          }
          const bool c0 = in0 && oe0 >= kAlphaThreshold;
          const bool c1 = in1 && oe1 >= kAlphaThreshold;
          const uint32_t hits = __ballot_sync(0xffffffffu, c0 || c1);
          if (hits == 0u) continue;
          const float4 col = s_col[j];
          float g[kRecordGradCount];
#pragma unroll
          for (int f = 0; f < kRecordGradCount; ++f) g[f] = 0.0f;
          const float dp0 = backward_pixel(q0, c0, oe0, e0, col, g);
          const float dp1 = backward_pixel(q1, c1, oe1, e1, col, g);
          // Moments of dp against the offsets: the two pixels share dx.
          const float dpy0 = dp0 * dy0, dpy1 = dp1 * dy1;
          g[kMDx] = dx * (dp0 + dp1);
          g[kMDy] = dpy0 + dpy1;
          g[kMDxx] = dx * g[kMDx];
          g[kMDxy] = dx * g[kMDy];
          g[kMDyy] = fmaf(dpy0, dy0, dpy1 * dy1);
          // Transposed warp sum: four halving exchanges leave lane l with a
          // partial sum of term (l >> 1) over 16 lanes, the last one adds the
          // other half; 16 shuffles instead of 5 per term.  (Direct shared
          // atomics for records that touch few lanes measured slower: the
          // lanes' adds to one record serialise.)
          float* dst = s_grad + j * kGradStride;
          float v[16];
#pragma unroll
          for (int f = 0; f < 16; ++f) v[f] = f < kRecordGradCount ? g[f] : 0.0f;
#pragma unroll
          for (int half = 8; half >= 1; half >>= 1) {
            const bool upper = (lane & (half * 2)) != 0;
#pragma unroll
            for (int i = 0; i < half; ++i) {
              const float send = upper ? v[i] : v[i + half];
              const float keep = upper ? v[i + half] : v[i];
              v[i] = keep + __shfl_xor_sync(0xffffffffu, send, half * 2);
            }
          }
          v[0] += __shfl_xor_sync(0xffffffffu, v[0], 1);
          const int term = lane >> 1;
          if ((lane & 1) == 0 && term < kRecordGradCount) atomicAdd(dst + term, v[0]);
        }
      }
    }
    __syncthreads();
    for (int j = tid; j < n; j += Geo::kThreads) {
      float g[kRecordGradCount];
      bool any = false;
#pragma unroll
      for (int f = 0; f < kRecordGradCount; ++f) {
        g[f] = s_grad[j * kGradStride + f];
        any |= g[f] != 0.0f;
      }
      if (!any) continue;
      // power = geo.z dx^2 + geo.w dx dy + cpo.x dy^2 with geo.z = -c0/2,
      // geo.w = -c1, cpo.x = -c2/2 and (dx, dy) = pixel - mean.
      const float4 geo = s_geo[j];
      const float cyy = s_cpo[j].x;
      const float d_mean_x = -(2.0f * geo.z * g[kMDx] + geo.w * g[kMDy]);
      const float d_mean_y = -(geo.w * g[kMDx] + 2.0f * cyy * g[kMDy]);
      float4* dst = p.record_grads + static_cast<int64_t>(p.values[lo + j]) * 3;
      atomicAdd(dst + 0, make_float4(d_mean_x, d_mean_y, -0.5f * g[kMDxx], -g[kMDxy]));
      atomicAdd(dst + 1, make_float4(-0.5f * g[kMDyy], g[kGOpacity], g[kGDepth], 0.0f));
      atomicAdd(dst + 2, make_float4(g[kGRed], g[kGGreen], g[kGBlue], 0.0f));
    }
    __syncthreads();
  }
}

template __global__ void composite_backward_kernel<4>(CompositeBackwardParams);
template __global__ void composite_backward_kernel<8>(CompositeBackwardParams);
template __global__ void composite_backward_kernel<16>(CompositeBackwardParams);

// ---------------------------------------------------------------------------
// Projection backward, one thread per Gaussian.
// ---------------------------------------------------------------------------
constexpr int kProjectBackwardThreads = 128;
// Real SH basis (the forward's constants) and its derivative with respect to
// the unit view direction (x, y, z), contracted with per-coefficient weights
// d_basis: returns sum_k d_basis[k] * d basis_k / d(x, y, z).
template <int kDegree>
__device__ __forceinline__ void sh_basis(float x, float y, float z, float* basis) {
  basis[0] = 0.28209479177387814f;
  if (kDegree >= 1) {
    basis[1] = fmul(-0.4886025119029199f, y);
    basis[2] = fmul(0.4886025119029199f, z);
    basis[3] = fmul(-0.4886025119029199f, x);
  }
  const float xx = fmul(x, x), yy = fmul(y, y), zz = fmul(z, z);
  const float xy = fmul(x, y), yz = fmul(y, z), xz = fmul(x, z);
  if (kDegree >= 2) {
    basis[4] = fmul(1.0925484305920792f, xy);
    basis[5] = fmul(-1.0925484305920792f, yz);
    basis[6] = fmul(0.31539156525252005f, fsub(fsub(fmul(2.0f, zz), xx), yy));
    basis[7] = fmul(-1.0925484305920792f, xz);
    basis[8] = fmul(0.5462742152960396f, fsub(xx, yy));
  }
  if (kDegree >= 3) {
    basis[9] = fmul(fmul(-0.5900435899266435f, y), fsub(fmul(3.0f, xx), yy));
    basis[10] = fmul(fmul(2.890611442640554f, xy), z);
    basis[11] = fmul(fmul(-0.4570457994644658f, y), fsub(fsub(fmul(4.0f, zz), xx), yy));
    basis[12] = fmul(fmul(0.3731763325901154f, z),
                     fsub(fsub(fmul(2.0f, zz), fmul(3.0f, xx)), fmul(3.0f, yy)));
    basis[13] = fmul(fmul(-0.4570457994644658f, x), fsub(fsub(fmul(4.0f, zz), xx), yy));
    basis[14] = fmul(fmul(1.445305721320277f, z), fsub(xx, yy));
    basis[15] = fmul(fmul(-0.5900435899266435f, x), fsub(xx, fmul(3.0f, yy)));
  }
}

template <int kDegree>
__device__ __forceinline__ void sh_direction_grad(float x, float y, float z, const float* db,
                                                  float* dn) {
  float gx = 0.0f, gy = 0.0f, gz = 0.0f;
  if (kDegree >= 1) {
    const float c1 = 0.4886025119029199f;
    gy -= c1 * db[1];
    gz += c1 * db[2];
    gx -= c1 * db[3];
  }
  if (kDegree >= 2) {
    const float c4 = 1.0925484305920792f, c6 = 0.31539156525252005f, c8 = 0.5462742152960396f;
    gx += c4 * y * db[4];
    gy += c4 * x * db[4];
    gy -= c4 * z * db[5];
    gz -= c4 * y * db[5];
    gx -= 2.0f * c6 * x * db[6];
    gy -= 2.0f * c6 * y * db[6];
    gz += 4.0f * c6 * z * db[6];
    gx -= c4 * z * db[7];
    gz -= c4 * x * db[7];
    gx += 2.0f * c8 * x * db[8];
    gy -= 2.0f * c8 * y * db[8];
  }
  if (kDegree >= 3) {
    const float c9 = 0.5900435899266435f, c10 = 2.890611442640554f, c11 = 0.4570457994644658f;
    const float c12 = 0.3731763325901154f, c14 = 1.445305721320277f;
    const float xx = x * x, yy = y * y, zz = z * z;
    gx -= 6.0f * c9 * x * y * db[9];
    gy -= 3.0f * c9 * (xx - yy) * db[9];
    gx += c10 * y * z * db[10];
    gy += c10 * x * z * db[10];
    gz += c10 * x * y * db[10];
    gx += 2.0f * c11 * x * y * db[11];
    gy -= c11 * (4.0f * zz - xx - 3.0f * yy) * db[11];
    gz -= 8.0f * c11 * y * z * db[11];
    gx -= 6.0f * c12 * x * z * db[12];
    gy -= 6.0f * c12 * y * z * db[12];
    gz += c12 * (6.0f * zz - 3.0f * xx - 3.0f * yy) * db[12];
    gx -= c11 * (4.0f * zz - 3.0f * xx - yy) * db[13];
    gy += 2.0f * c11 * x * y * db[13];
    gz -= 8.0f * c11 * x * z * db[13];
    gx += 2.0f * c14 * x * z * db[14];
    gy -= 2.0f * c14 * y * z * db[14];
    gz += c14 * (xx - yy) * db[14];
    gx -= 3.0f * c9 * (xx - yy) * db[15];
    gy += 6.0f * c9 * x * y * db[15];
  }
  dn[0] = gx;
  dn[1] = gy;
  dn[2] = gz;
}

template <int kShDegree>
__global__ void __launch_bounds__(kProjectBackwardThreads, 4) project_backward_kernel(ProjectBackwardParams p) {
  constexpr int kCount = kShDegree < 0 ? 1 : (kShDegree + 1) * (kShDegree + 1);
  constexpr int kFloats = kShDegree < 0 ? 3 : kCount * 3;
  constexpr int kVec = (kFloats + 3) / 4;
  constexpr int kPrefetch = 8;
  // Colour-coefficient sums live in shared memory as float4s, thread-major
  // (conflict-free): 48 accumulators in registers next to the coefficients
  // would cap the kernel at two CTAs per SM.
  __shared__ float4 s_dsh[kVec * kProjectBackwardThreads];
  const int64_t g = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (g >= p.gaussian_count) return;

  // Registered scene of g: offsets are non-decreasing, find the last slot
  // whose range starts at or before g and contains it.
  int scene = -1;
  {
    int lo = 0, hi = p.scene_count;  // answer in [lo, hi)
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (p.scene_offsets[mid] <= g) lo = mid; else hi = mid;
    }
    if (p.scene_count > 0 && p.scene_offsets[lo] <= g && g < p.scene_offsets[lo + 1]) scene = lo;
  }

  const float mx = p.means[g * 3 + 0], my = p.means[g * 3 + 1], mz = p.means[g * 3 + 2];
  const float s00 = p.covariances[g * 6 + 0], s01 = p.covariances[g * 6 + 1];
  const float s02 = p.covariances[g * 6 + 2], s11 = p.covariances[g * 6 + 3];
  const float s12 = p.covariances[g * 6 + 4], s22 = p.covariances[g * 6 + 5];
  // The Gaussian's colour coefficients are read again at each camera that
  // sees it (L1 hits after the first): held in registers across the loop
  // they capped the kernel at two CTAs per SM.
  const float* coef_row = p.features + g * p.feature_width;

  float dm[3] = {0.0f, 0.0f, 0.0f};
  float dcov[6] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
  float dop = 0.0f;
  float4* dsh = s_dsh + threadIdx.x;
#pragma unroll
  for (int i = 0; i < kVec; ++i) dsh[i * kProjectBackwardThreads] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);

  const CamPlan* plans = reinterpret_cast<const CamPlan*>(p.scratch + p.layout.plans);
  const CamConst* consts = reinterpret_cast<const CamConst*>(p.scratch + p.layout.cam_consts);
  for (int64_t a0 = 0; a0 < p.active_count && scene >= 0; a0 += kPrefetch) {
    // Record indices of up to kPrefetch cameras, all loads in flight at once.
    int32_t rr[kPrefetch];
#pragma unroll
    for (int u = 0; u < kPrefetch; ++u) {
      const int64_t a = a0 + u;
      rr[u] = -1;
      if (a < p.active_count) {
        const CamPlan& plan = plans[a];
        const int64_t local = g - plan.g_begin;
        if (plan.camera >= 0 && plan.scene_slot == scene && local >= 0 && local < plan.g_count &&
            local < p.record_map_stride) {
          rr[u] = p.record_map[a * p.record_map_stride + local];
        }
      }
    }
#pragma unroll 1
  for (int u = 0; u < kPrefetch; ++u) {
    const int32_t r = rr[u];
    if (r < 0) continue;
    const int64_t a = a0 + u;
    const float4 g0 = p.record_grads[static_cast<int64_t>(r) * 3 + 0];
    const float4 g1 = p.record_grads[static_cast<int64_t>(r) * 3 + 1];
    const float4 g2 = p.record_grads[static_cast<int64_t>(r) * 3 + 2];
    if (g0.x == 0.0f && g0.y == 0.0f && g0.z == 0.0f && g0.w == 0.0f && g1.x == 0.0f &&
        g1.y == 0.0f && g1.z == 0.0f && g2.x == 0.0f && g2.y == 0.0f && g2.z == 0.0f) {
      continue;
    }
    const CamConst c = consts[a];
    const float* R = c.r;

    // Forward recompute (the projection's operations).
    const float pz = ffma(R[8], mz, ffma(R[7], my, ffma(R[6], mx, c.t[2])));
    const float px = ffma(R[2], mz, ffma(R[1], my, ffma(R[0], mx, c.t[0])));
    const float py = ffma(R[5], mz, ffma(R[4], my, ffma(R[3], mx, c.t[1])));
    const float iz = fdiv(1.0f, pz);
    float tm[9];
#pragma unroll
    for (int row = 0; row < 3; ++row) {
      const float r0 = R[row * 3 + 0], r1 = R[row * 3 + 1], r2 = R[row * 3 + 2];
      tm[row * 3 + 0] = ffma(r2, s02, ffma(r1, s01, fmul(r0, s00)));
      tm[row * 3 + 1] = ffma(r2, s12, ffma(r1, s11, fmul(r0, s01)));
      tm[row * 3 + 2] = ffma(r2, s22, ffma(r1, s12, fmul(r0, s02)));
    }
    float cc3[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        cc3[i][j] = ffma(tm[i * 3 + 2], R[j * 3 + 2],
                         ffma(tm[i * 3 + 1], R[j * 3 + 1], fmul(tm[i * 3 + 0], R[j * 3 + 0])));
      }
    }
    const float c00 = cc3[0][0], c01 = cc3[0][1], c02 = cc3[0][2];
    const float c11 = cc3[1][1], c12 = cc3[1][2], c22 = cc3[2][2];
    const float tx = fmul(px, iz);
    const float ty = fmul(py, iz);
    const float ctx = fminf(c.lim_xp, fmaxf(-c.lim_xn, tx));
    const float cty = fminf(c.lim_yp, fmaxf(-c.lim_yn, ty));
    const float clx = fmul(pz, ctx);
    const float cly = fmul(pz, cty);
    const float iz2 = fmul(iz, iz);
    const float j00 = fmul(c.fx, iz);
    const float j02 = fmul(fmul(-c.fx, clx), iz2);
    const float j11 = fmul(c.fy, iz);
    const float j12 = fmul(fmul(-c.fy, cly), iz2);
    const float a_raw =
        ffma(fmul(j02, j02), c22, ffma(fmul(fmul(2.0f, j00), j02), c02, fmul(fmul(j00, j00), c00)));
    const float b = ffma(fmul(j02, j12), c22,
                         ffma(fmul(j02, j11), c12, ffma(fmul(j00, j12), c02, fmul(fmul(j00, j11), c01))));
    const float c_raw =
        ffma(fmul(j12, j12), c22, ffma(fmul(fmul(2.0f, j11), j12), c12, fmul(fmul(j11, j11), c11)));
    const float ca = fadd(a_raw, p.cov_eps);
    const float cc = fadd(c_raw, p.cov_eps);
    const float det = ffma(ca, cc, -fmul(b, b));

    // conic = (cc, -b, a) / det  ->  2D covariance (a, b, cc).
    const float id = 1.0f / det;
    const float id2 = id * id;
    const float d_det = -(g0.z * cc - g0.w * b + g1.x * ca) * id2;
    const float d_a = g1.x * id + d_det * cc;
    const float d_c = g0.z * id + d_det * ca;
    const float d_b = -g0.w * id - 2.0f * b * d_det;
    // 2D covariance -> camera covariance and Jacobian.
    float dc[3][3];
    dc[0][0] = d_a * j00 * j00;
    dc[0][1] = 0.5f * d_b * j00 * j11;
    dc[0][2] = d_a * j00 * j02 + 0.5f * d_b * j00 * j12;
    dc[1][1] = d_c * j11 * j11;
    dc[1][2] = 0.5f * d_b * j02 * j11 + d_c * j11 * j12;
    dc[2][2] = d_a * j02 * j02 + d_b * j02 * j12 + d_c * j12 * j12;
    dc[1][0] = dc[0][1];
    dc[2][0] = dc[0][2];
    dc[2][1] = dc[1][2];
    const float d_j00 = d_a * (2.0f * j00 * c00 + 2.0f * j02 * c02) + d_b * (j11 * c01 + j12 * c02);
    const float d_j02 = d_a * (2.0f * j00 * c02 + 2.0f * j02 * c22) + d_b * (j11 * c12 + j12 * c22);
    const float d_j11 = d_b * (j00 * c01 + j02 * c12) + d_c * (2.0f * j11 * c11 + 2.0f * j12 * c12);
    const float d_j12 = d_b * (j00 * c02 + j02 * c22) + d_c * (2.0f * j11 * c12 + 2.0f * j12 * c22);
    float d_iz = d_j00 * c.fx + d_j11 * c.fy - 2.0f * c.fx * clx * iz * d_j02 -
                 2.0f * c.fy * cly * iz * d_j12;
    const float d_clx = -c.fx * iz2 * d_j02;
    const float d_cly = -c.fy * iz2 * d_j12;
    float d_px = 0.0f, d_py = 0.0f, d_pz = g1.z;  // depth = pz
    // Mean: u = fx px / pz + cx, v = fy py / pz + cy.
    d_px += g0.x * c.fx * iz;
    d_py += g0.y * c.fy * iz;
    d_iz += g0.x * c.fx * px + g0.y * c.fy * py;
    // Clamped Jacobian point: clx = pz * clamp(px / pz).
    if (tx >= -c.lim_xn && tx <= c.lim_xp) d_px += d_clx; else d_pz += d_clx * ctx;
    if (ty >= -c.lim_yn && ty <= c.lim_yp) d_py += d_cly; else d_pz += d_cly * cty;
    d_pz -= d_iz * iz * iz;

    // Colour.
    if (kShDegree < 0) {
      float4 d = dsh[0];
      d.x += g2.x;
      d.y += g2.y;
      d.z += g2.z;
      dsh[0] = d;
    } else {
      const float dvx = ffma(R[6], pz, ffma(R[3], py, fmul(R[0], px)));
      const float dvy = ffma(R[7], pz, ffma(R[4], py, fmul(R[1], px)));
      const float dvz = ffma(R[8], pz, ffma(R[5], py, fmul(R[2], px)));
      const float inv = fdiv(1.0f, fsqrt(ffma(dvz, dvz, ffma(dvy, dvy, fmul(dvx, dvx)))));
      const float x = fmul(dvx, inv), y = fmul(dvy, inv), z = fmul(dvz, inv);
      float basis[16];
      sh_basis<kShDegree < 0 ? 0 : kShDegree>(x, y, z, basis);
      float coef[kVec * 4];
      if (p.vector_feature_loads) {
#pragma unroll
        for (int i = 0; i < kVec; ++i) {
          const float4 v = __ldg(reinterpret_cast<const float4*>(coef_row) + i);
          coef[4 * i + 0] = v.x;
          coef[4 * i + 1] = v.y;
          coef[4 * i + 2] = v.z;
          coef[4 * i + 3] = v.w;
        }
      } else {
#pragma unroll
        for (int f = 0; f < kVec * 4; ++f) coef[f] = f < kFloats ? __ldg(coef_row + f) : 0.0f;
      }
      float acc[3] = {0.0f, 0.0f, 0.0f};
#pragma unroll
      for (int k = 0; k < kCount; ++k) {
#pragma unroll
        for (int ch = 0; ch < 3; ++ch) {
          acc[ch] = k == 0 ? fmul(basis[0], coef[ch]) : ffma(basis[k], coef[k * 3 + ch], acc[ch]);
        }
      }
      const float drgb[3] = {fadd(acc[0], 0.5f) > 0.0f ? g2.x : 0.0f,
                             fadd(acc[1], 0.5f) > 0.0f ? g2.y : 0.0f,
                             fadd(acc[2], 0.5f) > 0.0f ? g2.z : 0.0f};
#pragma unroll
      for (int i = 0; i < kVec; ++i) {
        float4 d = dsh[i * kProjectBackwardThreads];
        float* dv = reinterpret_cast<float*>(&d);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const int f = 4 * i + q;
          if (f < kFloats) dv[q] = fmaf(basis[f / 3], drgb[f % 3], dv[q]);
        }
        dsh[i * kProjectBackwardThreads] = d;
      }
      if (kShDegree >= 1) {
        float db[16];
#pragma unroll
        for (int k = 0; k < kCount; ++k) {
          db[k] = coef[k * 3 + 0] * drgb[0] + coef[k * 3 + 1] * drgb[1] + coef[k * 3 + 2] * drgb[2];
        }
        float dn[3];
        sh_direction_grad<kShDegree < 0 ? 0 : kShDegree>(x, y, z, db, dn);
        const float ndot = x * dn[0] + y * dn[1] + z * dn[2];
        const float ddx = (dn[0] - x * ndot) * inv;
        const float ddy = (dn[1] - y * ndot) * inv;
        const float ddz = (dn[2] - z * ndot) * inv;
        // direction = R^T p
        d_px += R[0] * ddx + R[1] * ddy + R[2] * ddz;
        d_py += R[3] * ddx + R[4] * ddy + R[5] * ddz;
        d_pz += R[6] * ddx + R[7] * ddy + R[8] * ddz;
      }
    }
    dop += g1.y;
    // p = R m + t.
    dm[0] += R[0] * d_px + R[3] * d_py + R[6] * d_pz;
    dm[1] += R[1] * d_px + R[4] * d_py + R[7] * d_pz;
    dm[2] += R[2] * d_px + R[5] * d_py + R[8] * d_pz;
    // Camera covariance = R Sigma R^T  ->  dSigma = R^T dC R (symmetric).
    float t3[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        t3[i][j] = dc[i][0] * R[0 * 3 + j] + dc[i][1] * R[1 * 3 + j] + dc[i][2] * R[2 * 3 + j];
      }
    }
    float gs[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        gs[i][j] = R[0 * 3 + i] * t3[0][j] + R[1 * 3 + i] * t3[1][j] + R[2 * 3 + i] * t3[2][j];
      }
    }
    dcov[0] += gs[0][0];
    dcov[1] += gs[0][1] + gs[1][0];
    dcov[2] += gs[0][2] + gs[2][0];
    dcov[3] += gs[1][1];
    dcov[4] += gs[1][2] + gs[2][1];
    dcov[5] += gs[2][2];
  }
  }

  // Activations.  Opacity: o = sigmoid(logit).
  const float o = p.opacities[g];
  p.d_opacity_logits[g] = dop * o * (1.0f - o);
  // Covariance Sigma = M M^T with M = R(q) diag(s), s = exp(log_scale).
  float qr[9];
  float qinv;
  const float qw = p.rotations[g * 4 + 0], qx = p.rotations[g * 4 + 1];
  const float qy = p.rotations[g * 4 + 2], qz = p.rotations[g * 4 + 3];
  quaternion_rotation(qw, qx, qy, qz, qr, &qinv);
  const float sc[3] = {vexp(clamp_exp_arg(p.log_scales[g * 3 + 0])),
                       vexp(clamp_exp_arg(p.log_scales[g * 3 + 1])),
                       vexp(clamp_exp_arg(p.log_scales[g * 3 + 2]))};
  const float G[3][3] = {{dcov[0], 0.5f * dcov[1], 0.5f * dcov[2]},
                         {0.5f * dcov[1], dcov[3], 0.5f * dcov[4]},
                         {0.5f * dcov[2], 0.5f * dcov[4], dcov[5]}};
  float dR[9];
  float ds[3] = {0.0f, 0.0f, 0.0f};
#pragma unroll
  for (int i = 0; i < 3; ++i) {
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      // dM_ij = 2 (G M)_ij, M_kj = R_kj s_j.
      const float dmij =
          2.0f * (G[i][0] * qr[0 * 3 + j] + G[i][1] * qr[1 * 3 + j] + G[i][2] * qr[2 * 3 + j]) * sc[j];
      dR[i * 3 + j] = dmij * sc[j];
      ds[j] += dmij * qr[i * 3 + j];
    }
  }
#pragma unroll
  for (int j = 0; j < 3; ++j) p.d_log_scales[g * 3 + j] = ds[j] * sc[j];
  // Rotation matrix of the normalised quaternion (w, x, y, z).
  const float w = qw * qinv, x = qx * qinv, y = qy * qinv, z = qz * qinv;
  const float dw = 2.0f * (-z * dR[1] + y * dR[2] + z * dR[3] - x * dR[5] - y * dR[6] + x * dR[7]);
  const float dx = 2.0f * (y * dR[1] + z * dR[2] + y * dR[3] - 2.0f * x * dR[4] - w * dR[5] +
                           z * dR[6] + w * dR[7] - 2.0f * x * dR[8]);
  const float dy = 2.0f * (-2.0f * y * dR[0] + x * dR[1] + w * dR[2] + x * dR[3] + z * dR[5] -
                           w * dR[6] + z * dR[7] - 2.0f * y * dR[8]);
  const float dz = 2.0f * (-2.0f * z * dR[0] - w * dR[1] + x * dR[2] + w * dR[3] - 2.0f * z * dR[4] +
                           y * dR[5] + x * dR[6] + y * dR[7]);
  // Normalisation q / |q|.
  const float ndot = w * dw + x * dx + y * dy + z * dz;
  p.d_rotations[g * 4 + 0] = (dw - w * ndot) * qinv;
  p.d_rotations[g * 4 + 1] = (dx - x * ndot) * qinv;
  p.d_rotations[g * 4 + 2] = (dy - y * ndot) * qinv;
  p.d_rotations[g * 4 + 3] = (dz - z * ndot) * qinv;
#pragma unroll
  for (int k = 0; k < 3; ++k) p.d_means[g * 3 + k] = dm[k];
  float* dfeat = p.d_features + g * p.feature_width;
#pragma unroll
  for (int i = 0; i < kVec; ++i) {
    const float4 d = dsh[i * kProjectBackwardThreads];
    const float dv[4] = {d.x, d.y, d.z, d.w};
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      if (4 * i + q < kFloats) dfeat[4 * i + q] = dv[q];
    }
  }
  for (int64_t k = kFloats; k < p.feature_width; ++k) dfeat[k] = 0.0f;
}

template __global__ void project_backward_kernel<-1>(ProjectBackwardParams);
template __global__ void project_backward_kernel<0>(ProjectBackwardParams);
template __global__ void project_backward_kernel<1>(ProjectBackwardParams);
template __global__ void project_backward_kernel<2>(ProjectBackwardParams);
template __global__ void project_backward_kernel<3>(ProjectBackwardParams);

}  // namespace vgr
