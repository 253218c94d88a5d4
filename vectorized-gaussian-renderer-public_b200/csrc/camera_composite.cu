// Fused front-to-back RGB/depth/alpha/semantic compositor.
//
// Equation of src/isaacsim_gaussian_renderer/native/renderer_cuda.cu:1973-2305
// (screen-space path): per pixel, records in (depth, Gaussian id) order,
// alpha = min(0.99, o exp(power)) for -20 <= power <= 0 and alpha >= 1/255,
// stop before blending a record whose next transmittance is <= 1e-4, weight
// w = T alpha, RGB and depth accumulate w-weighted, alpha = 1 - T,
// depth = sum(w z) / alpha (or +inf), semantic = label of the largest single
// w (the earliest wins ties) or -1 when alpha < semantic_min_alpha.
//
// B200 structure: one CTA per (camera, tile); records are staged in batches
// of 256 through shared memory together with an 8-bit mask of the warps whose
// 8x4 pixel block the record's conservative alpha footprint touches.  Each
// warp walks only its own records with __ballot_sync over the masks, skips
// exp for pixels beyond a per-record quadratic-form bound, and retires as a
// unit once all of its pixels have terminated; the CTA stops staging when
// __syncthreads_count reports no live pixel.
#include "vgr_kernels.h"

namespace vgr {

template <int kTile>
struct CompositeGeometry {
  static constexpr int kPixels = kTile * kTile;
  static constexpr int kBlockW = kTile < 8 ? kTile : 8;          // warp sub-block width
  static constexpr int kBlockH = (32 / kBlockW) < kTile ? (32 / kBlockW) : kTile;
  static constexpr int kWarpsX = kTile / kBlockW;
  static constexpr int kWarpsY = kTile / kBlockH;
  static constexpr int kWarps = kWarpsX * kWarpsY;
  static constexpr int kThreads = kWarps * 32;
};

constexpr int kCompositeBatch = 256;

template <int kTile, bool kFull>
__global__ void __launch_bounds__(CompositeGeometry<kTile>::kThreads)
    composite_kernel(CompositeParams p) {
  using Geo = CompositeGeometry<kTile>;
  __shared__ float4 s_a[kCompositeBatch];
  __shared__ float4 s_b[kCompositeBatch];
  __shared__ float4 s_c[kCompositeBatch];
  __shared__ float s_qmax[kCompositeBatch];
  __shared__ uint32_t s_mask[kCompositeBatch];
  __shared__ int64_t s_sem[kFull ? kCompositeBatch : 1];

  const CamPlan* plans = reinterpret_cast<const CamPlan*>(p.scratch + p.layout.plans);
  const int64_t* tile_prefix = reinterpret_cast<const int64_t*>(p.scratch + p.layout.tile_prefix);

  // Work item -> active slot.  Slots are dense in [0, A) and every slot's
  // tiles are contiguous; tile_prefix is monotone, so search it.
  const int64_t item = blockIdx.x;
  const int64_t total = tile_prefix[p.active_count];
  if (item >= total) return;
  int64_t lo = 0, hi = p.active_count;  // tile_prefix[lo] <= item < tile_prefix[hi]
  {
    // Uniform batches: direct guess first.
    const int64_t tpi = p.tiles_per_camera_hint;
    if (tpi > 0) {
      const int64_t guess = item / tpi;
      if (guess < p.active_count && tile_prefix[guess] <= item && item < tile_prefix[guess + 1]) {
        lo = guess;
        hi = guess + 1;
      }
    }
    while (hi - lo > 1) {
      const int64_t mid = (lo + hi) >> 1;
      if (tile_prefix[mid] <= item) lo = mid; else hi = mid;
    }
  }
  const CamPlan plan = plans[lo];
  const int64_t local_tile = item - tile_prefix[lo];
  const int tile_y = static_cast<int>(local_tile / plan.tiles_x);
  const int tile_x = static_cast<int>(local_tile - static_cast<int64_t>(tile_y) * plan.tiles_x);
  const int64_t global_tile = plan.tile_base + local_tile;

  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  const int warp_x = warp % Geo::kWarpsX;
  const int warp_y = warp / Geo::kWarpsX;
  const int lx = lane % Geo::kBlockW;
  const int ly = lane / Geo::kBlockW;
  const int pixel_x = tile_x * kTile + warp_x * Geo::kBlockW + lx;
  const int pixel_y = tile_y * kTile + warp_y * Geo::kBlockH + ly;
  const bool valid = ly < Geo::kBlockH && pixel_x < plan.width && pixel_y < plan.height;
  const float cx = fadd(static_cast<float>(pixel_x), 0.5f);
  const float cy = fadd(static_cast<float>(pixel_y), 0.5f);

  float transmittance = 1.0f;
  float acc_r = 0.0f, acc_g = 0.0f, acc_b = 0.0f, acc_depth = 0.0f;
  float best_weight = -1.0f;
  int64_t best_semantic = -1;
  bool done = !valid;
  bool warp_done = __all_sync(0xffffffffu, done);

  const int64_t range_start = p.tile_starts[global_tile];
  const int64_t range_end = p.tile_ends[global_tile];
  const float tile_x0 = static_cast<float>(tile_x * kTile);
  const float tile_y0 = static_cast<float>(tile_y * kTile);

  if (range_start >= 0 && range_end > range_start) {
    for (int64_t chunk = range_start; chunk < range_end; chunk += kCompositeBatch) {
      const int n = static_cast<int>(min(static_cast<int64_t>(kCompositeBatch), range_end - chunk));
      for (int j = tid; j < n; j += Geo::kThreads) {
        const int32_t v = p.values[chunk + j];
        const Record rec = p.records[v];
        s_a[j] = rec.a;
        s_b[j] = rec.b;
        s_c[j] = rec.c;
        if (kFull) s_sem[j] = p.semantic_ids[__float_as_int(rec.b.w)];
        const float o = rec.b.y;
        s_qmax[j] = fminf(40.0f, 2.0f * __logf(255.0f * o)) * 1.001f + 1.0e-3f;
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
        s_mask[j] = mask;
      }
      __syncthreads();
      if (!warp_done) {
        for (int base = 0; base < n && !warp_done; base += 32) {
          const uint32_t m = (base + lane < n) ? s_mask[base + lane] : 0u;
          uint32_t bits = __ballot_sync(0xffffffffu, (m >> warp) & 1u);
          while (bits) {
            const int j = base + __ffs(bits) - 1;
            bits &= bits - 1;
            if (!done) {
              const float4 ra = s_a[j];
              const float conic2 = s_b[j].x;
              const float dx = fsub(cx, ra.x);
              const float dy = fsub(cy, ra.y);
              const float q = ffma(fmul(conic2, dy), dy,
                                   ffma(fmul(fmul(2.0f, ra.w), dx), dy, fmul(fmul(ra.z, dx), dx)));
              if (q <= s_qmax[j]) {
                const float power = fmul(-0.5f, q);
                if (!(power > 0.0f || power < -20.0f)) {
                  const float4 rb = s_b[j];
                  const float alpha = fminf(kMaxAlpha, fmul(rb.y, vexp(power)));
                  if (alpha >= kAlphaThreshold) {
                    const float next_t = fmul(transmittance, fsub(1.0f, alpha));
                    if (next_t <= kTransmittanceThreshold) {
                      done = true;
                    } else {
                      const float w = fmul(transmittance, alpha);
                      const float4 rc = s_c[j];
                      acc_r = ffma(w, rc.x, acc_r);
                      acc_g = ffma(w, rc.y, acc_g);
                      acc_b = ffma(w, rc.z, acc_b);
                      if (kFull) {
                        acc_depth = ffma(w, rb.z, acc_depth);
                        if (w > best_weight) {
                          best_weight = w;
                          best_semantic = s_sem[j];
                        }
                      }
                      transmittance = next_t;
                    }
                  }
                }
              }
            }
            if (__all_sync(0xffffffffu, done)) {
              warp_done = true;
              break;
            }
          }
        }
      }
      if (__syncthreads_count(!done) == 0) break;
    }
  }

  if (!valid) return;
  const int64_t pixel = plan.pixel_base + static_cast<int64_t>(pixel_y) * plan.width + pixel_x;
  const float out_alpha = fsub(1.0f, transmittance);
  if (p.output_srgb) {
    acc_r = linear_to_srgb(acc_r);
    acc_g = linear_to_srgb(acc_g);
    acc_b = linear_to_srgb(acc_b);
  }
  p.rgb[pixel * 3 + 0] = acc_r;
  p.rgb[pixel * 3 + 1] = acc_g;
  p.rgb[pixel * 3 + 2] = acc_b;
  if (kFull) {
    p.alpha[pixel] = out_alpha;
    p.depth[pixel] = out_alpha > 1.0e-8f ? fdiv(acc_depth, out_alpha) : __int_as_float(0x7f800000);
    p.semantic[pixel] =
        (best_weight >= 0.0f && out_alpha >= p.semantic_min_alpha) ? best_semantic : -1;
  }
}

template __global__ void composite_kernel<4, false>(CompositeParams);
template __global__ void composite_kernel<4, true>(CompositeParams);
template __global__ void composite_kernel<8, false>(CompositeParams);
template __global__ void composite_kernel<8, true>(CompositeParams);
template __global__ void composite_kernel<16, false>(CompositeParams);
template __global__ void composite_kernel<16, true>(CompositeParams);

}  // namespace vgr
