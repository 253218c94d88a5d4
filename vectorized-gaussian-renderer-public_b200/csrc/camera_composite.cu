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
// over the masks, skips exp beyond a per-record quadratic-form bound (each
// pixel tests its own power: a warp-wide "any pixel in range" test in front
// of the blends cost more in votes and branches than the colour load it
// saved, 7 % of the compositor's time), and retires once all of its pixels
// have terminated; the CTA stops staging when
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

// One work item (one (camera, tile), or with kSplit > 1 one kTile-pixel
// quadrant of a (kSplit * kTile)-pixel tile whose sorted list the quadrants
// share); every exit is CTA-uniform.  kPix pixels per thread: rows y and
// y + kLaneRows of the warp block when two.
template <int kTile, bool kFull, bool kTrain, int kSplit, int kPix, int kBatch>
__device__ __forceinline__ void composite_item(const CompositeParams& p, int64_t work,
                                               float4* s_geo, float4* s_cpo, float4* s_col,
                                               uint32_t* s_mask) {
  using Geo = CompositeGeometry<kTile, kPix>;
  CamPlan plan;
  int64_t local_tile;
  const int64_t item = work / (kSplit * kSplit);
  const int quad = static_cast<int>(work - item * (kSplit * kSplit));
  if (!locate_tile(p.scratch, p.layout, p.active_count, p.tiles_per_camera_hint, item, plan,
                   local_tile)) {
    return;
  }
  const int bin_y = static_cast<int>(local_tile / plan.tiles_x);
  const int bin_x = static_cast<int>(local_tile - static_cast<int64_t>(bin_y) * plan.tiles_x);
  const int64_t global_tile = plan.tile_base + local_tile;
  const int tile_x = bin_x * kSplit + quad % kSplit;  // in kTile units
  const int tile_y = bin_y * kSplit + quad / kSplit;
  if (tile_x * kTile >= plan.width || tile_y * kTile >= plan.height) return;

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
  const float kNaN = __int_as_float(0x7fc00000);
  const float cx = fadd(static_cast<float>(pixel_x), 0.5f);
  bool valid[kPix];
  float cy[kPix];
  PixelState s[kPix];
  bool all_done = true;
#pragma unroll
  for (int q = 0; q < kPix; ++q) {
    const int pixel_y = pixel_y0 + q * Geo::kLaneRows;
    valid[q] = lane_used && pixel_x < plan.width && pixel_y < plan.height;
    cy[q] = valid[q] ? fadd(static_cast<float>(pixel_y), 0.5f) : kNaN;
    s[q] = PixelState{1.0f, 0.0f, 0.0f, 0.0f, 0.0f, -1.0f, 0, 0, !valid[q]};
    all_done = all_done && s[q].done;
  }
  bool warp_done = __all_sync(0xffffffffu, all_done);

  const int64_t range_start = p.tile_starts[global_tile];
  const int64_t range_end = p.tile_ends[global_tile];
  const float tile_x0 = static_cast<float>(tile_x * kTile);
  const float tile_y0 = static_cast<float>(tile_y * kTile);

  if (range_start >= 0 && range_end > range_start) {
    for (int64_t chunk = range_start; chunk < range_end; chunk += kBatch) {
      const int n = static_cast<int>(min(static_cast<int64_t>(kBatch), range_end - chunk));
      for (int j = tid; j < n; j += Geo::kThreads) {
        stage_composite_record<kTile, kPix>(p.records[p.values[chunk + j]], tile_x0, tile_y0, s_geo[j],
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
            const float4 col = s_col[j];
#pragma unroll
            for (int q = 0; q < kPix; ++q) {
              const float dy = fsub(cy[q], geo.y);
              const float pw = ffma(fmul(cpo.x, dy), dy, ffma(bdx, dy, adx));
              blend<kFull, kTrain>(s[q], cy[q], pw, cpo.y, cpo.z, chunk_pos + j, col);
            }
          }
          all_done = true;
#pragma unroll
          for (int q = 0; q < kPix; ++q) all_done = all_done && s[q].done;
          warp_done = __all_sync(0xffffffffu, all_done);
        }
      }
      bool live = false;
#pragma unroll
      for (int q = 0; q < kPix; ++q) live = live || !s[q].done;
      if (__syncthreads_count(live) == 0) break;
    }
  }

#pragma unroll
  for (int q = 0; q < kPix; ++q) {
    if (valid[q]) write_pixel<kFull, kTrain>(p, plan, pixel_x, pixel_y0 + q * Geo::kLaneRows, s[q]);
  }
}

// Resident CTAs per SM of each compositor shape: forward 16-pixel tiles in
// the default shape keep three quarters of the SM's threads resident (a
// 40-register cap: the loop is latency- and issue-bound, and the extra warps
// measured 2.6 % faster than half occupancy at 64 registers); the
// half-occupancy shape keeps half, and so do the other tile sizes.
template <int kTile, bool kTrain, int kShape>
struct CompositeOccupancy {
  static constexpr int kThreads = CompositeGeometry<kTile, CompositeShape<kShape>::kPix>::kThreads;
  static constexpr bool kThreeQuarters = kTile == 16 && !kTrain && kShape != kShapeHalfOccupancy;
  static constexpr int kBlocks = kThreeQuarters ? 2048 / kThreads * 3 / 4 : 2048 / kThreads / 2;
};

// One CTA per work item, or (p.persistent) a resident grid whose CTAs take
// work items from a device queue (ScratchHeader::composite_queue, zeroed by
// the camera setup) until every (camera, tile) of the frame is done: no
// CTA is launched for the grid's empty tail, and a CTA that finishes a cheap
// tile immediately takes the next one.
template <int kTile, bool kFull, bool kTrain, int kSplit, int kShape>
__global__ void __launch_bounds__(CompositeOccupancy<kTile, kTrain, kShape>::kThreads,
                                  CompositeOccupancy<kTile, kTrain, kShape>::kBlocks)
    composite_kernel(CompositeParams p) {
  constexpr int kPix = CompositeShape<kShape>::kPix;
  // Records staged per batch: the half-occupancy shape of 16-pixel tiles has
  // the shared memory for 512 (fewer batch barriers: 11.0 -> 10.9 ms on the
  // ragged frame), the others 256 (one-warp CTAs of 8-pixel tiles need their
  // residency more than fewer barriers).
  constexpr int kBatch = kTile == 16 && kShape == kShapeHalfOccupancy ? 2 * kCompositeBatch : kCompositeBatch;
  __shared__ float4 s_geo[kBatch];  // mean_x, mean_y, -conic_xx/2, -conic_xy
  __shared__ float4 s_cpo[kBatch];  // -conic_yy/2, lo, opacity, -
  __shared__ float4 s_col[kBatch];  // r, g, b, depth
  __shared__ uint32_t s_mask[kBatch];
  __shared__ uint32_t s_item;
  if (!p.persistent) {
    composite_item<kTile, kFull, kTrain, kSplit, kPix, kBatch>(p, blockIdx.x, s_geo, s_cpo, s_col, s_mask);
    return;
  }
  ScratchHeader* header = reinterpret_cast<ScratchHeader*>(p.scratch + p.layout.header);
  const int64_t* tile_prefix = reinterpret_cast<const int64_t*>(p.scratch + p.layout.tile_prefix);
  const int64_t total = tile_prefix[p.active_count] * (kSplit * kSplit);
  while (true) {
    if (threadIdx.x == 0) s_item = atomicAdd(&header->composite_queue, 1u);
    __syncthreads();
    const int64_t item = s_item;
    if (item >= total) break;
    composite_item<kTile, kFull, kTrain, kSplit, kPix, kBatch>(p, item, s_geo, s_cpo, s_col, s_mask);
    __syncthreads();  // shared staging and s_item are reused by the next item
  }
}

// ---------------------------------------------------------------------------
// Exact-ray compositor (renderer_cuda.cu:203-245 and 2190-2270): every pixel
// casts the camera ray d = (nx, ny, 1), nx = (x + 0.5 - cx) / fx, and each
// record in (depth, Gaussian id) order contributes alpha = min(1, o
// exp(-m^2/2)) with m^2 = max(0, m^T P m - (d^T P m)^2 / d^T P d), the
// squared Mahalanobis distance from the mean to the ray, for m^2 <= sigma^2.
// No 1/255 cut and no 0.99 clamp; the record that takes T to <= 1e-4 is
// blended and then the pixel stops.  Same CTA and pixel layout as the
// screen-space compositor, without its warp footprint masks (the record's
// ellipse is the tile cover itself).  A terminated pixel's ray_y becomes NaN,
// so every later d^T P d is NaN and fails the > 0 test.
// Each record is evaluated only at pixels inside the box of its ray ellipse
// (radius + 1 px around the ellipse centre, record c.w): outside it the exact
// m^2 exceeds sigma^2, so this drops only float-cancellation artefacts, and it
// lets each warp skip the records whose box misses its 8x8 block.
// ---------------------------------------------------------------------------
template <bool kFull>
__device__ __forceinline__ void blend_ray(PixelState& s, float& ray_y, float alpha, int32_t pos,
                                          const float4& col) {
  const float next_t = fmul(s.transmittance, fsub(1.0f, alpha));
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
  s.transmittance = next_t;
  if (next_t <= kTransmittanceThreshold) {
    s.done = true;
    ray_y = __int_as_float(0x7fc00000);
  }
}

// alpha of one record on one ray (0 when it does not contribute); t_*
// carry the ray_x products shared by the thread's two pixels.
__device__ __forceinline__ float ray_alpha(const float4& p0, const float4& p1, const float4& p2,
                                           float ray_x, float ray_y, float t_xx, float t_xy,
                                           float t_x, float t_m, float s2) {
  if (!(ray_y == ray_y)) return 0.0f;  // terminated or outside the record's box
  // d^T P d = P00 x^2 + 2 P01 x y + 2 P02 x + P11 y^2 + 2 P12 y + P22
  const float rpr = fadd(
      ffma(fmul(2.0f, p1.x), ray_y,
           ffma(fmul(p0.w, ray_y), ray_y, ffma(t_x, ray_x, ffma(t_xy, ray_y, t_xx)))),
      p1.y);
  if (!(rpr > 0.0f)) return 0.0f;
  const float rpm = fadd(ffma(ray_y, p1.w, t_m), p2.x);
  const float rpm2 = fmul(rpm, rpm);
  if (rpr < 1.0e30f) {
    // Fast rejection: the approximate quotient is within 3 ulp of the IEEE
    // one, so with this margin a rejected ray has the exact m^2 > sigma^2 too.
    const float qa = __fdividef(rpm2, rpr);
    if (fsub(p2.y, qa) > s2 + 1.0e-6f * (fabsf(qa) + s2)) return 0.0f;
  }
  const float m2 = fmaxf(0.0f, fsub(p2.y, fdiv(rpm2, rpr)));
  // m^2 > 174 would take exp below the float range of the polynomial exp:
  // alpha < 2e-38, no contribution.
  if (!(m2 <= s2) || !(m2 <= 174.0f)) return 0.0f;
  return fminf(1.0f, fmul(p2.z, vexp(fmul(-0.5f, m2))));
}

// kSplit: CTAs per bin side.  A 32-pixel bin (16-pixel tiles in exact-ray
// mode) is composited by four 16-pixel CTAs that read the same sorted list:
// smaller CTAs wait less at the batch barriers, and each pixel still sees
// its bin's records in the same order.
template <int kTile, bool kFull, int kSplit>
__global__ void __launch_bounds__(CompositeGeometry<kTile>::kThreads,
                                  2048 / CompositeGeometry<kTile>::kThreads / 2)
    composite_ray_kernel(CompositeParams p) {
  using Geo = CompositeGeometry<kTile>;
  __shared__ float4 s_p0[kCompositeBatch];   // P00, P01, P02, P11
  __shared__ float4 s_p1[kCompositeBatch];   // P12, P22, Pm0, Pm1
  __shared__ float4 s_p2[kCompositeBatch];   // Pm2, mPm, opacity, -
  __shared__ float4 s_col[kCompositeBatch];  // r, g, b, depth
  __shared__ float4 s_box[kCompositeBatch];  // centre x, centre y, half-extent x, y
  __shared__ uint32_t s_mask[kCompositeBatch];
  CamPlan plan;
  int64_t local_tile;
  const int64_t item = blockIdx.x / (kSplit * kSplit);
  const int quad = static_cast<int>(blockIdx.x - item * (kSplit * kSplit));
  if (!locate_tile(p.scratch, p.layout, p.active_count, p.tiles_per_camera_hint, item, plan,
                   local_tile)) {
    return;
  }
  const int bin_y = static_cast<int>(local_tile / plan.tiles_x);
  const int bin_x = static_cast<int>(local_tile - static_cast<int64_t>(bin_y) * plan.tiles_x);
  const int64_t global_tile = plan.tile_base + local_tile;
  const int origin_x = (bin_x * kSplit + quad % kSplit) * kTile;
  const int origin_y = (bin_y * kSplit + quad / kSplit) * kTile;
  if (origin_x >= plan.width || origin_y >= plan.height) return;  // quadrant past the image edge

  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  const int lx = lane % Geo::kBlockW;
  const int ly = lane / Geo::kBlockW;
  const bool lane_used = ly < Geo::kLaneRows;
  const int pixel_x = origin_x + (warp % Geo::kWarpsX) * Geo::kBlockW + lx;
  const int pixel_y0 = origin_y + (warp / Geo::kWarpsX) * Geo::kBlockH + ly;
  const int pixel_y1 = pixel_y0 + Geo::kLaneRows;
  const bool valid0 = lane_used && pixel_x < plan.width && pixel_y0 < plan.height;
  const bool valid1 = lane_used && pixel_x < plan.width && pixel_y1 < plan.height;
  const float kNaN = __int_as_float(0x7fc00000);
  const float* in = p.intrinsics + static_cast<int64_t>(plan.camera) * 9;
  const float fx = in[0], cxi = in[2], fy = in[4], cyi = in[5];
  const float cx = fadd(static_cast<float>(pixel_x), 0.5f);
  const float cy0 = fadd(static_cast<float>(pixel_y0), 0.5f);
  const float cy1 = fadd(static_cast<float>(pixel_y1), 0.5f);
  const float ray_x = fdiv(fsub(cx, cxi), fx);
  float ray_y0 = valid0 ? fdiv(fsub(cy0, cyi), fy) : kNaN;
  float ray_y1 = valid1 ? fdiv(fsub(cy1, cyi), fy) : kNaN;
  const float tile_x0 = static_cast<float>(origin_x);
  const float tile_y0 = static_cast<float>(origin_y);
  const float s2 = fmul(p.support_sigma, p.support_sigma);

  PixelState s0{1.0f, 0.0f, 0.0f, 0.0f, 0.0f, -1.0f, 0, 0, !valid0};
  PixelState s1{1.0f, 0.0f, 0.0f, 0.0f, 0.0f, -1.0f, 0, 0, !valid1};
  bool warp_done = __all_sync(0xffffffffu, s0.done && s1.done);

  const int64_t range_start = p.tile_starts[global_tile];
  const int64_t range_end = p.tile_ends[global_tile];
  if (range_start >= 0 && range_end > range_start) {
    for (int64_t chunk = range_start; chunk < range_end; chunk += kCompositeBatch) {
      const int n = static_cast<int>(min(static_cast<int64_t>(kCompositeBatch), range_end - chunk));
      for (int j = tid; j < n; j += Geo::kThreads) {
        const int32_t r = p.values[chunk + j];
        const Record& rec = p.records[r];
        const float4 e2 = p.ray_ext[static_cast<int64_t>(r) * 3 + 2];
        s_p0[j] = p.ray_ext[static_cast<int64_t>(r) * 3 + 0];
        s_p1[j] = p.ray_ext[static_cast<int64_t>(r) * 3 + 1];
        s_p2[j] = make_float4(e2.x, e2.y, rec.b.y, 0.0f);
        s_col[j] = make_float4(rec.c.x, rec.c.y, rec.c.z, rec.b.z);
        const uint32_t bits = __float_as_uint(rec.c.w);
        const float hx = (bits & 0xffffu) >= 32767u ? __int_as_float(0x7f800000)
                                                    : static_cast<float>(bits & 0xffffu);
        const float hy = (bits >> 16) >= 32767u ? __int_as_float(0x7f800000) : static_cast<float>(bits >> 16);
        s_box[j] = make_float4(rec.a.x, rec.a.y, hx, hy);
        uint32_t mask = 0;
#pragma unroll
        for (int w = 0; w < Geo::kWarps; ++w) {
          const float bx0 = tile_x0 + static_cast<float>((w % Geo::kWarpsX) * Geo::kBlockW) + 0.5f;
          const float by0 = tile_y0 + static_cast<float>((w / Geo::kWarpsX) * Geo::kBlockH) + 0.5f;
          const float bx1 = bx0 + static_cast<float>(Geo::kBlockW - 1);
          const float by1 = by0 + static_cast<float>(Geo::kBlockH - 1);
          const bool hit = !(fsub(bx0, rec.a.x) > hx || fsub(rec.a.x, bx1) > hx ||
                             fsub(by0, rec.a.y) > hy || fsub(rec.a.y, by1) > hy);
          mask |= hit ? (1u << w) : 0u;
        }
        s_mask[j] = mask;
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
            const float4 box = s_box[j];
            const bool in_x = !(fabsf(fsub(cx, box.x)) > box.z);
            const float y0 = (in_x && !(fabsf(fsub(cy0, box.y)) > box.w)) ? ray_y0 : kNaN;
            const float y1 = (in_x && !(fabsf(fsub(cy1, box.y)) > box.w)) ? ray_y1 : kNaN;
            if (!(y0 == y0) && !(y1 == y1)) continue;
            const float4 p0 = s_p0[j];
            const float4 p1 = s_p1[j];
            const float4 p2 = s_p2[j];
            const float t_xx = fmul(fmul(p0.x, ray_x), ray_x);
            const float t_xy = fmul(fmul(2.0f, p0.y), ray_x);
            const float t_x = fmul(2.0f, p0.z);
            const float t_m = fmul(ray_x, p1.z);
            const float a0 = ray_alpha(p0, p1, p2, ray_x, y0, t_xx, t_xy, t_x, t_m, s2);
            const float a1 = ray_alpha(p0, p1, p2, ray_x, y1, t_xx, t_xy, t_x, t_m, s2);
            if (a0 > 0.0f || a1 > 0.0f) {
              const float4 col = s_col[j];
              if (a0 > 0.0f) blend_ray<kFull>(s0, ray_y0, a0, chunk_pos + j, col);
              if (a1 > 0.0f) blend_ray<kFull>(s1, ray_y1, a1, chunk_pos + j, col);
            }
          }
          warp_done = __all_sync(0xffffffffu, s0.done && s1.done);
        }
      }
      if (__syncthreads_count(!(s0.done && s1.done)) == 0) break;
    }
  }
  if (valid0) write_pixel<kFull, false>(p, plan, pixel_x, pixel_y0, s0);
  if (valid1) write_pixel<kFull, false>(p, plan, pixel_x, pixel_y1, s1);
}

template __global__ void composite_ray_kernel<4, false, 1>(CompositeParams);
template __global__ void composite_ray_kernel<4, true, 1>(CompositeParams);
template __global__ void composite_ray_kernel<8, false, 1>(CompositeParams);
template __global__ void composite_ray_kernel<8, true, 1>(CompositeParams);
template __global__ void composite_ray_kernel<16, false, 1>(CompositeParams);
template __global__ void composite_ray_kernel<16, true, 1>(CompositeParams);
template __global__ void composite_ray_kernel<16, false, 2>(CompositeParams);
template __global__ void composite_ray_kernel<16, true, 2>(CompositeParams);

#define VGR_COMPOSITE_SHAPES(TILE, FULL, SPLIT)                                      \
  template __global__ void composite_kernel<TILE, FULL, false, SPLIT, kShapeDefault>(CompositeParams); \
  template __global__ void composite_kernel<TILE, FULL, false, SPLIT, kShapeOnePixel>(CompositeParams); \
  template __global__ void composite_kernel<TILE, FULL, false, SPLIT, kShapeHalfOccupancy>(CompositeParams);
template __global__ void composite_kernel<4, false, false, 1, kShapeDefault>(CompositeParams);
template __global__ void composite_kernel<4, true, false, 1, kShapeDefault>(CompositeParams);
VGR_COMPOSITE_SHAPES(8, false, 1)
VGR_COMPOSITE_SHAPES(8, true, 1)
VGR_COMPOSITE_SHAPES(16, false, 1)
VGR_COMPOSITE_SHAPES(16, true, 1)
VGR_COMPOSITE_SHAPES(16, false, 2)
VGR_COMPOSITE_SHAPES(16, true, 2)
#undef VGR_COMPOSITE_SHAPES
template __global__ void composite_kernel<4, true, true, 1, kShapeDefault>(CompositeParams);
template __global__ void composite_kernel<8, true, true, 1, kShapeDefault>(CompositeParams);
template __global__ void composite_kernel<16, true, true, 1, kShapeDefault>(CompositeParams);

}  // namespace vgr
