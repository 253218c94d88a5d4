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
// B200 structure: one CTA per (camera, tile); each thread owns two pixels of
// one column (rows y and y + kLaneRows) so the per-record work shared by the
// pair (shared-memory loads, dx, a*dx*dx, 2b*dx, loop control) is paid once.
// Records are staged in batches of 256 through shared memory together with a
// mask of the warps whose 8x8-pixel block the record's conservative alpha
// footprint touches; each warp walks only its records with __ballot_sync
// over the masks, skips exp beyond a per-record quadratic-form bound, and
// retires once all of its pixels have terminated; the CTA stops staging when
// __syncthreads_count reports no live pixel.  The semantic label is resolved
// once per pixel at the end from the sorted position of its largest weight.
#include "vgr_kernels.h"

namespace vgr {

// Per-pixel accumulation.  A pixel that terminates gets a NaN row coordinate,
// so every later power evaluates to NaN and fails the range test: the hot
// path never tests `done`, which only drives the warp and CTA exits.
struct PixelState {
  float transmittance;
  float r, g, b, depth;
  float best_weight;
  int32_t best_pos;  // sorted position of the largest single weight
  int32_t last;      // training: sorted position one past the last blended record
  bool done;
};

// One record on one pixel.  power = -q/2 evaluated from conic terms scaled by
// -1/2 (exact: scaling by a power of two commutes with rounding), lo =
// max(-qmax/2, -20) merges the conservative q bound with the reference's
// power >= -20 cut, so the test below is the reference's
// `power <= 0 && power >= -20` restricted to records that can reach 1/255.
template <bool kFull, bool kTrain>
__device__ __forceinline__ void blend(PixelState& s, float& cy, float power, float lo, float o,
                                      int32_t pos, const float4& col) {
  if (!(power >= lo && power <= 0.0f)) return;
  const float alpha = fminf(kMaxAlpha, fmul(o, vexp(power)));
  if (!(alpha >= kAlphaThreshold)) return;
  const float next_t = fmul(s.transmittance, fsub(1.0f, alpha));
  if (next_t <= kTransmittanceThreshold) {
    s.done = true;
    cy = __int_as_float(0x7fc00000);
    return;
  }
  const float w = fmul(s.transmittance, alpha);
  s.r = ffma(w, col.x, s.r);
  s.g = ffma(w, col.y, s.g);
  s.b = ffma(w, col.z, s.b);
  if (kFull) {
    s.depth = ffma(w, col.w, s.depth);
    if (w > s.best_weight) {
      s.best_weight = w;
      s.best_pos = pos;
    }
  }
  if (kTrain) s.last = pos + 1;
  s.transmittance = next_t;
}

template <bool kFull, bool kTrain>
__device__ __forceinline__ void write_pixel(const CompositeParams& p, const CamPlan& plan, int x,
                                            int y, PixelState& s) {
  const int64_t pixel = plan.pixel_base + static_cast<int64_t>(y) * plan.width + x;
  const float out_alpha = fsub(1.0f, s.transmittance);
  if (p.output_srgb) {
    s.r = linear_to_srgb(s.r);
    s.g = linear_to_srgb(s.g);
    s.b = linear_to_srgb(s.b);
  }
  p.rgb[pixel * 3 + 0] = s.r;
  p.rgb[pixel * 3 + 1] = s.g;
  p.rgb[pixel * 3 + 2] = s.b;
  if (kFull) {
    p.alpha[pixel] = out_alpha;
    p.depth[pixel] = out_alpha > 1.0e-8f ? fdiv(s.depth, out_alpha) : __int_as_float(0x7f800000);
    int64_t semantic = -1;
    if (s.best_weight >= 0.0f && out_alpha >= p.semantic_min_alpha) {
      const Record& rec = p.records[p.values[s.best_pos]];
      semantic = p.semantic_ids[__float_as_int(rec.b.w)];
    }
    p.semantic[pixel] = semantic;
  }
  if (kTrain) {
    p.final_transmittance[pixel] = s.transmittance;
    p.last_position[pixel] = s.last;
  }
}

// One work item (one (camera, tile)); every exit is CTA-uniform.
template <int kTile, bool kFull, bool kTrain>
__device__ __forceinline__ void composite_item(const CompositeParams& p, int64_t item,
                                               float4* s_geo, float4* s_cpo, float4* s_col,
                                               uint32_t* s_mask) {
  using Geo = CompositeGeometry<kTile>;
  CamPlan plan;
  int64_t local_tile;
  if (!locate_tile(p.scratch, p.layout, p.active_count, p.tiles_per_camera_hint, item, plan,
                   local_tile)) {
    return;
  }
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
  const bool lane_used = ly < Geo::kLaneRows;
  const int pixel_x = tile_x * kTile + warp_x * Geo::kBlockW + lx;
  const int pixel_y0 = tile_y * kTile + warp_y * Geo::kBlockH + ly;
  const int pixel_y1 = pixel_y0 + Geo::kLaneRows;
  const bool valid0 = lane_used && pixel_x < plan.width && pixel_y0 < plan.height;
  const bool valid1 = lane_used && pixel_x < plan.width && pixel_y1 < plan.height;
  const float kNaN = __int_as_float(0x7fc00000);
  const float cx = fadd(static_cast<float>(pixel_x), 0.5f);
  float cy0 = valid0 ? fadd(static_cast<float>(pixel_y0), 0.5f) : kNaN;
  float cy1 = valid1 ? fadd(static_cast<float>(pixel_y1), 0.5f) : kNaN;

  PixelState s0{1.0f, 0.0f, 0.0f, 0.0f, 0.0f, -1.0f, 0, 0, !valid0};
  PixelState s1{1.0f, 0.0f, 0.0f, 0.0f, 0.0f, -1.0f, 0, 0, !valid1};
  bool warp_done = __all_sync(0xffffffffu, s0.done && s1.done);

  const int64_t range_start = p.tile_starts[global_tile];
  const int64_t range_end = p.tile_ends[global_tile];
  const float tile_x0 = static_cast<float>(tile_x * kTile);
  const float tile_y0 = static_cast<float>(tile_y * kTile);

  if (range_start >= 0 && range_end > range_start) {
    for (int64_t chunk = range_start; chunk < range_end; chunk += kCompositeBatch) {
      const int n = static_cast<int>(min(static_cast<int64_t>(kCompositeBatch), range_end - chunk));
      for (int j = tid; j < n; j += Geo::kThreads) {
        stage_composite_record<kTile>(p.records[p.values[chunk + j]], tile_x0, tile_y0, s_geo[j],
                                      s_cpo[j], s_col[j], s_mask[j]);
      }
      __syncthreads();
      if (!warp_done) {
        const int32_t chunk_pos = static_cast<int32_t>(chunk);
        for (int base = 0; base < n && !warp_done; base += 32) {
          const uint32_t m = (base + lane < n) ? s_mask[base + lane] : 0u;
          uint32_t bits = __ballot_sync(0xffffffffu, (m >> warp) & 1u);
          while (bits) {
            const int j = base + __ffs(bits) - 1;
            bits &= bits - 1;
            const float4 geo = s_geo[j];
            const float4 cpo = s_cpo[j];
            const float dx = fsub(cx, geo.x);
            const float adx = fmul(fmul(geo.z, dx), dx);
            const float bdx = fmul(geo.w, dx);
            const float dy0 = fsub(cy0, geo.y);
            const float dy1 = fsub(cy1, geo.y);
            const float p0 = ffma(fmul(cpo.x, dy0), dy0, ffma(bdx, dy0, adx));
            const float p1 = ffma(fmul(cpo.x, dy1), dy1, ffma(bdx, dy1, adx));
            const bool in0 = p0 >= cpo.y && p0 <= 0.0f;
            const bool in1 = p1 >= cpo.y && p1 <= 0.0f;
            if (in0 || in1) {
              const float4 col = s_col[j];
              blend<kFull, kTrain>(s0, cy0, p0, cpo.y, cpo.z, chunk_pos + j, col);
              blend<kFull, kTrain>(s1, cy1, p1, cpo.y, cpo.z, chunk_pos + j, col);
            }
          }
          warp_done = __all_sync(0xffffffffu, s0.done && s1.done);
        }
      }
      if (__syncthreads_count(!(s0.done && s1.done)) == 0) break;
    }
  }

  if (valid0) write_pixel<kFull, kTrain>(p, plan, pixel_x, pixel_y0, s0);
  if (valid1) write_pixel<kFull, kTrain>(p, plan, pixel_x, pixel_y1, s1);
}

// One CTA per work item, or (p.persistent) a resident grid whose CTAs take
// work items from a device queue (ScratchHeader::composite_queue, zeroed by
// the camera setup) until every (camera, tile) of the frame is done: no
// CTA is launched for the grid's empty tail, and a CTA that finishes a cheap
// tile immediately takes the next one.
template <int kTile, bool kFull, bool kTrain>
__global__ void __launch_bounds__(CompositeGeometry<kTile>::kThreads,
                                  2048 / CompositeGeometry<kTile>::kThreads / 2)
    composite_kernel(CompositeParams p) {
  __shared__ float4 s_geo[kCompositeBatch];  // mean_x, mean_y, -conic_xx/2, -conic_xy
  __shared__ float4 s_cpo[kCompositeBatch];  // -conic_yy/2, lo, opacity, -
  __shared__ float4 s_col[kCompositeBatch];  // r, g, b, depth
  __shared__ uint32_t s_mask[kCompositeBatch];
  __shared__ uint32_t s_item;
  if (!p.persistent) {
    composite_item<kTile, kFull, kTrain>(p, blockIdx.x, s_geo, s_cpo, s_col, s_mask);
    return;
  }
  ScratchHeader* header = reinterpret_cast<ScratchHeader*>(p.scratch + p.layout.header);
  const int64_t* tile_prefix = reinterpret_cast<const int64_t*>(p.scratch + p.layout.tile_prefix);
  const int64_t total = tile_prefix[p.active_count];
  while (true) {
    if (threadIdx.x == 0) s_item = atomicAdd(&header->composite_queue, 1u);
    __syncthreads();
    const int64_t item = s_item;
    if (item >= total) break;
    composite_item<kTile, kFull, kTrain>(p, item, s_geo, s_cpo, s_col, s_mask);
    __syncthreads();  // shared staging and s_item are reused by the next item
  }
}

template __global__ void composite_kernel<4, false, false>(CompositeParams);
template __global__ void composite_kernel<4, true, false>(CompositeParams);
template __global__ void composite_kernel<8, false, false>(CompositeParams);
template __global__ void composite_kernel<8, true, false>(CompositeParams);
template __global__ void composite_kernel<16, false, false>(CompositeParams);
template __global__ void composite_kernel<16, true, false>(CompositeParams);
template __global__ void composite_kernel<4, true, true>(CompositeParams);
template __global__ void composite_kernel<8, true, true>(CompositeParams);
template __global__ void composite_kernel<16, true, true>(CompositeParams);

}  // namespace vgr
