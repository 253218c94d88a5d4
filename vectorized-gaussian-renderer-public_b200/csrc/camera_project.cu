// Camera setup, EWA projection, ordered compaction and tile emission.
//
// Follows the reference camera equation of
// src/isaacsim_gaussian_renderer/native/renderer_cuda.cu:287-490 (projection,
// cull, radius, conic) and :1691-1829 (tile cover and key), restructured for
// B200: one persistent launch walks virtual blocks of kProjectChunk
// (camera, Gaussian) tasks handed out by an atomic ticket, compacts visible
// records and their tile intersections in task order within the block,
// reserves the block's output ranges with one atomic per kind (blocks never
// wait on each other, whatever their cost), and emits the keys cooperatively
// from shared memory so every store is coalesced, counting each tile's keys
// for the bucket sort.  There is no host round trip: the totals stay on the
// device for the sort.
#include "vgr_camera.cuh"
#include "vgr_kernels.h"

namespace vgr {

// ---------------------------------------------------------------------------
// Camera setup: one CTA builds the per-active-camera plans and projection
// constants, the exclusive prefix of tiles over active cameras (the
// compositor's work list), and zeroes counters and queue tickets so the frame
// needs no host memset.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(1024) camera_setup_kernel(SetupParams p) {
  __shared__ int64_t s_warp_sums[32];
  __shared__ int64_t s_carry;
  ScratchHeader* header = reinterpret_cast<ScratchHeader*>(p.scratch + p.layout.header);
  CamPlan* plans = reinterpret_cast<CamPlan*>(p.scratch + p.layout.plans);
  CamConst* cam_consts = reinterpret_cast<CamConst*>(p.scratch + p.layout.cam_consts);
  int64_t* tile_prefix = reinterpret_cast<int64_t*>(p.scratch + p.layout.tile_prefix);
  const int tid = threadIdx.x;
  if (tid < 32) {
    reinterpret_cast<uint32_t*>(header)[tid] = 0u;
  }
  if (p.reset_counters && tid < 5) {
    p.counters[tid] = 0;
  }
  if (p.reset_counters) {
    uint32_t* hist = reinterpret_cast<uint32_t*>(p.scratch + p.layout.sort_hist);
    for (int i = tid; i < kMaxSortPasses * kRadixBins; i += blockDim.x) hist[i] = 0u;
  }
  if (tid == 0) s_carry = 0;
  __syncthreads();

  for (int64_t base = 0; base < p.active_count; base += blockDim.x) {
    const int64_t a = base + tid;
    int64_t tiles = 0;
    if (a < p.active_count) {
      CamPlan plan;
      const int64_t cam64 = p.active_ids ? p.active_ids[a] : a;
      plan.camera = -1;
      plan.scene_slot = -1;
      plan.g_begin = 0;
      plan.g_count = 0;
      plan.width = 0;
      plan.height = 0;
      plan.tiles_x = 0;
      plan.tiles_y = 0;
      plan.tile_base = 0;
      plan.pixel_base = 0;
      if (cam64 >= 0 && cam64 < p.batch) {
        const int cam = static_cast<int>(cam64);
        plan.camera = cam;
        const int64_t requested = p.camera_scene_ids[cam];
        for (int s = 0; s < p.scene_count; ++s) {
          if (p.registered_scene_ids[s] == requested) {
            plan.scene_slot = s;
            break;
          }
        }
        if (plan.scene_slot >= 0) {
          plan.g_begin = p.scene_offsets[plan.scene_slot];
          plan.g_count = p.scene_offsets[plan.scene_slot + 1] - plan.g_begin;
          if (plan.g_count < 0) plan.g_count = 0;
        }
        if (p.widths) {
          plan.width = p.widths[cam];
          plan.height = p.heights[cam];
          plan.tile_base = p.tile_offsets[cam];
          plan.pixel_base = p.pixel_offsets[cam];
        } else {
          plan.width = p.width;
          plan.height = p.height;
        }
        plan.tiles_x = (plan.width + p.tile_size - 1) / p.tile_size;
        plan.tiles_y = (plan.height + p.tile_size - 1) / p.tile_size;
        if (!p.widths) {
          plan.tile_base = static_cast<int64_t>(cam) * plan.tiles_x * plan.tiles_y;
          plan.pixel_base = static_cast<int64_t>(cam) * plan.width * plan.height;
        }
        tiles = static_cast<int64_t>(plan.tiles_x) * plan.tiles_y;
        make_cam_const(p.viewmats + cam * 16, p.env_xforms + cam * 16, p.intrinsics + cam * 9,
                       plan.width, plan.height, cam_consts + a);
      }
      plans[a] = plan;
    }
    // Block-wide exclusive scan of tiles.
    int64_t v = tiles;
    const int lane = tid & 31;
    const int warp = tid >> 5;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int64_t n = __shfl_up_sync(0xffffffffu, v, o);
      if (lane >= o) v += n;
    }
    if (lane == 31) s_warp_sums[warp] = v;
    __syncthreads();
    if (warp == 0) {
      int64_t w = (lane < static_cast<int>(blockDim.x >> 5)) ? s_warp_sums[lane] : 0;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int64_t n = __shfl_up_sync(0xffffffffu, w, o);
        if (lane >= o) w += n;
      }
      s_warp_sums[lane] = w;
    }
    __syncthreads();
    const int64_t warp_prefix = warp > 0 ? s_warp_sums[warp - 1] : 0;
    const int64_t inclusive = s_carry + warp_prefix + v;
    if (a < p.active_count) tile_prefix[a] = inclusive - tiles;
    __syncthreads();
    if (tid == static_cast<int>(blockDim.x) - 1) s_carry = inclusive;
    __syncthreads();
  }
  if (tid == 0) tile_prefix[p.active_count] = s_carry;
}

struct Projected {
  float mean_x, mean_y;
  float conic0, conic1, conic2;
  float opacity;
  float depth;
  float cov_a, cov_b, cov_c;
  float px, py, pz;
  int radius_x, radius_y;
  // Exact-ray mode: camera-space precision (upper triangle), precision times
  // the camera-space mean, and mean^T precision mean, rounded from double.
  float prec[6], prec_mean[3], mean_prec_mean;
};

// EWA projection of one Gaussian (renderer_cuda.cu:287-490 screen-space path;
// with kRay the exact-ray additions of renderer_cuda.cu:795-948).
template <bool kRay>
__device__ __forceinline__ bool project_gaussian(const float* __restrict__ means,
                                                 const float* __restrict__ covariances,
                                                 const float* __restrict__ opacities,
                                                 int64_t g, const CamConst& c, float near_plane,
                                                 float far_plane, float support_sigma,
                                                 float cov_eps, bool antialiased,
                                                 Projected* out) {
  float o = opacities[g];
  if (!(o >= kAlphaThreshold)) return false;
  const float mx = means[g * 3 + 0];
  const float my = means[g * 3 + 1];
  const float mz = means[g * 3 + 2];
  const float pz = ffma(c.r[8], mz, ffma(c.r[7], my, ffma(c.r[6], mx, c.t[2])));
  if (pz < near_plane || pz > far_plane) return false;
  const float px = ffma(c.r[2], mz, ffma(c.r[1], my, ffma(c.r[0], mx, c.t[0])));
  const float py = ffma(c.r[5], mz, ffma(c.r[4], my, ffma(c.r[3], mx, c.t[1])));
  const float iz = fdiv(1.0f, pz);
  const float u = ffma(fmul(c.fx, px), iz, c.cx);
  const float v = ffma(fmul(c.fy, py), iz, c.cy);

  const float* s = covariances + g * 6;
  const float s00 = s[0], s01 = s[1], s02 = s[2], s11 = s[3], s12 = s[4], s22 = s[5];
  float tm[9];
#pragma unroll
  for (int row = 0; row < 3; ++row) {
    const float r0 = c.r[row * 3 + 0], r1 = c.r[row * 3 + 1], r2 = c.r[row * 3 + 2];
    tm[row * 3 + 0] = ffma(r2, s02, ffma(r1, s01, fmul(r0, s00)));
    tm[row * 3 + 1] = ffma(r2, s12, ffma(r1, s11, fmul(r0, s01)));
    tm[row * 3 + 2] = ffma(r2, s22, ffma(r1, s12, fmul(r0, s02)));
  }
#define VGR_COV(i, j) \
  ffma(tm[i * 3 + 2], c.r[j * 3 + 2], ffma(tm[i * 3 + 1], c.r[j * 3 + 1], fmul(tm[i * 3 + 0], c.r[j * 3 + 0])))
  const float c00 = VGR_COV(0, 0);
  const float c01 = VGR_COV(0, 1);
  const float c02 = VGR_COV(0, 2);
  const float c11 = VGR_COV(1, 1);
  const float c12 = VGR_COV(1, 2);
  const float c22 = VGR_COV(2, 2);
#undef VGR_COV

  const float tx = fmul(px, iz);
  const float ty = fmul(py, iz);
  const float clx = fmul(pz, fminf(c.lim_xp, fmaxf(-c.lim_xn, tx)));
  const float cly = fmul(pz, fminf(c.lim_yp, fmaxf(-c.lim_yn, ty)));
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
  const float a = fadd(a_raw, cov_eps);
  const float cc = fadd(c_raw, cov_eps);
  const float det = ffma(a, cc, -fmul(b, b));
  if (!(det > 0.0f)) return false;
  if (antialiased) {
    const float det_raw = ffma(a_raw, c_raw, -fmul(b, b));
    const float floor2 = fmul(kMinAntialiasCompensation, kMinAntialiasCompensation);
    const float comp = fsqrt(fmaxf(floor2, fdiv(det_raw, det)));
    o = fmul(o, comp);
    if (!(o >= kAlphaThreshold)) return false;
  }
  const float ext_o = fsqrt(fmul(2.0f, vlog(fdiv(o, kAlphaThreshold))));
  const float ext = fminf(support_sigma, ext_o);
  int rx = ceil_radius(fmul(ext, fsqrt(a)));
  int ry = ceil_radius(fmul(ext, fsqrt(cc)));
  if (rx <= 0 && ry <= 0) return false;
  float cull_x = u, cull_y = v;
  if (kRay) {
    // Precision of the camera-space covariance, and the image-plane ellipse
    // where a pixel ray's Mahalanobis distance to the mean is at most sigma:
    // the rays x = (nx, ny, 1) t with (m^T P d)^2 / (d^T P d) >= m^T P m -
    // sigma^2 form the conic d^T K d <= 0, K = (m^T P m - sigma^2) P -
    // (P m)(P m)^T, whose centre and extents (in normalised coordinates)
    // give the record's cull centre and tile radius.  A degenerate or
    // unbounded ellipse falls back to the whole image.
    const double d00 = c00, d01 = c01, d02 = c02, d11 = c11, d12 = c12, d22 = c22;
    const double det3 = dadd(dsub(dmul(d00, dsub(dmul(d11, d22), dmul(d12, d12))),
                                  dmul(d01, dsub(dmul(d01, d22), dmul(d02, d12)))),
                             dmul(d02, dsub(dmul(d01, d12), dmul(d02, d11))));
    if (!(det3 > 1.0e-48)) return false;
    const double inv3 = ddiv(1.0, det3);
    const double p00 = dmul(dsub(dmul(d11, d22), dmul(d12, d12)), inv3);
    const double p01 = dmul(dsub(dmul(d02, d12), dmul(d01, d22)), inv3);
    const double p02 = dmul(dsub(dmul(d01, d12), dmul(d02, d11)), inv3);
    const double p11 = dmul(dsub(dmul(d00, d22), dmul(d02, d02)), inv3);
    const double p12 = dmul(dsub(dmul(d01, d02), dmul(d00, d12)), inv3);
    const double p22 = dmul(dsub(dmul(d00, d11), dmul(d01, d01)), inv3);
    const double x = px, y = py, z = pz;
    const double m0 = dadd(dadd(dmul(p00, x), dmul(p01, y)), dmul(p02, z));
    const double m1 = dadd(dadd(dmul(p01, x), dmul(p11, y)), dmul(p12, z));
    const double m2 = dadd(dadd(dmul(p02, x), dmul(p12, y)), dmul(p22, z));
    const double mpm = dadd(dadd(dmul(x, m0), dmul(y, m1)), dmul(z, m2));
    out->prec[0] = static_cast<float>(p00);
    out->prec[1] = static_cast<float>(p01);
    out->prec[2] = static_cast<float>(p02);
    out->prec[3] = static_cast<float>(p11);
    out->prec[4] = static_cast<float>(p12);
    out->prec[5] = static_cast<float>(p22);
    out->prec_mean[0] = static_cast<float>(m0);
    out->prec_mean[1] = static_cast<float>(m1);
    out->prec_mean[2] = static_cast<float>(m2);
    out->mean_prec_mean = static_cast<float>(mpm);
    const double sg = static_cast<double>(support_sigma);
    const double q = dsub(mpm, dmul(sg, sg));
    const double k00 = dsub(dmul(q, p00), dmul(m0, m0));
    const double k01 = dsub(dmul(q, p01), dmul(m0, m1));
    const double k02 = dsub(dmul(q, p02), dmul(m0, m2));
    const double k11 = dsub(dmul(q, p11), dmul(m1, m1));
    const double k12 = dsub(dmul(q, p12), dmul(m1, m2));
    const double k22 = dsub(dmul(q, p22), dmul(m2, m2));
    const double kdet = dsub(dmul(k00, k11), dmul(k01, k01));
    bool finite = false;
    if (k00 > 0.0 && kdet > 0.0) {
      const double ikd = ddiv(1.0, kdet);
      const double cxn = dmul(dsub(dmul(k01, k12), dmul(k11, k02)), ikd);
      const double cyn = dmul(dsub(dmul(k01, k02), dmul(k00, k12)), ikd);
      const double scale = -dadd(dadd(k22, dmul(k02, cxn)), dmul(k12, cyn));
      if (scale > 0.0) {
        const double exn = dsqrt(dmul(dmul(scale, k11), ikd));
        const double eyn = dsqrt(dmul(dmul(scale, k00), ikd));
        const double cmx = dadd(dmul(static_cast<double>(c.fx), cxn), static_cast<double>(c.cx));
        const double cmy = dadd(dmul(static_cast<double>(c.fy), cyn), static_cast<double>(c.cy));
        cull_x = static_cast<float>(cmx);
        cull_y = static_cast<float>(cmy);
        rx = max(1, static_cast<int>(ceilf(static_cast<float>(dmul(fabs(static_cast<double>(c.fx)), exn)))));
        ry = max(1, static_cast<int>(ceilf(static_cast<float>(dmul(fabs(static_cast<double>(c.fy)), eyn)))));
        finite = isfinite(cmx) && isfinite(cmy) && isfinite(exn) && isfinite(eyn);
      }
    }
    if (!finite) {
      const int full = max(static_cast<int>(c.width), static_cast<int>(c.height));
      cull_x = fmul(0.5f, c.width);
      cull_y = fmul(0.5f, c.height);
      rx = full;
      ry = full;
    }
  }
  const float frx = static_cast<float>(rx);
  const float fry = static_cast<float>(ry);
  if (fadd(cull_x, frx) <= 0.0f || fadd(cull_y, fry) <= 0.0f || fsub(cull_x, frx) >= c.width ||
      fsub(cull_y, fry) >= c.height) {
    return false;
  }
  const float idet = fdiv(1.0f, det);
  out->mean_x = cull_x;
  out->mean_y = cull_y;
  out->conic0 = fmul(cc, idet);
  out->conic1 = fmul(-b, idet);
  out->conic2 = fmul(a, idet);
  out->opacity = fminf(fmaxf(o, 0.0f), 1.0f);
  out->depth = pz;
  out->cov_a = a;
  out->cov_b = b;
  out->cov_c = cc;
  out->px = px;
  out->py = py;
  out->pz = pz;
  out->radius_x = rx;
  out->radius_y = ry;
  return true;
}

// Real spherical harmonics through degree 3 (the basis and constants of the
// 3D Gaussian Splatting reference implementation, as used by gsplat), view
// direction from the camera centre to the mean in object space, +0.5 offset,
// clamped at zero.  coeffs is [(d+1)^2, 3], coefficient-major.  The row is
// fetched in 256-bit loads with wide_loads (rows 32-byte aligned and padded
// to a multiple of eight floats), else as float4s with vector_loads (16 bytes
// and four floats), otherwise as scalars; the sums are the same.
template <int kDegree>
__device__ __forceinline__ void eval_sh(const float* __restrict__ row, bool wide_loads, bool vector_loads,
                                        const CamConst& c, float px, float py, float pz,
                                        float* rgb) {
  constexpr int kCount = (kDegree + 1) * (kDegree + 1);
  constexpr int kFloats = kCount * 3;
  constexpr int kVectors = (kFloats + 3) / 4;
  constexpr int kOctets = (kFloats + 7) / 8;
  float dx = ffma(c.r[6], pz, ffma(c.r[3], py, fmul(c.r[0], px)));
  float dy = ffma(c.r[7], pz, ffma(c.r[4], py, fmul(c.r[1], px)));
  float dz = ffma(c.r[8], pz, ffma(c.r[5], py, fmul(c.r[2], px)));
  const float inv = fdiv(1.0f, fsqrt(ffma(dz, dz, ffma(dy, dy, fmul(dx, dx)))));
  const float x = fmul(dx, inv), y = fmul(dy, inv), z = fmul(dz, inv);
  float basis[16];
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
  // Coefficients are consumed as they arrive: float f of the row is channel
  // f % 3 of coefficient f / 3, and each channel's terms are added in
  // ascending coefficient order (the same sum as a per-channel loop).
  float acc[3] = {0.0f, 0.0f, 0.0f};
  auto take = [&](int f, float v) {
    const int k = f / 3;
    const int ch = f - 3 * k;
    if (k >= kCount) return;
    acc[ch] = k == 0 ? fmul(basis[0], v) : ffma(basis[k], v, acc[ch]);
  };
  if (wide_loads) {
#pragma unroll
    for (int i = 0; i < kOctets; ++i) {
      float v[8];
      ldg8(row + 8 * i, v);
#pragma unroll
      for (int k = 0; k < 8; ++k) take(8 * i + k, v[k]);
    }
  } else if (vector_loads) {
    const float4* row4 = reinterpret_cast<const float4*>(row);
#pragma unroll
    for (int i = 0; i < kVectors; ++i) {
      const float4 v = __ldg(row4 + i);
      take(4 * i + 0, v.x);
      take(4 * i + 1, v.y);
      take(4 * i + 2, v.z);
      take(4 * i + 3, v.w);
    }
  } else {
#pragma unroll
    for (int f = 0; f < kFloats; ++f) take(f, __ldg(row + f));
  }
#pragma unroll
  for (int ch = 0; ch < 3; ++ch) rgb[ch] = fmaxf(fadd(acc[ch], 0.5f), 0.0f);
}

// Conservative half-extents (pixels) of the region where a record can reach
// alpha >= 1/255 before the power < -20 cut: the ellipse q(d) <= t with
// t = min(40, 2 ln(255 o)).  Used only to skip warps that cannot be touched;
// ill-conditioned footprints report an infinite box (no skipping).
__device__ __forceinline__ uint32_t footprint_box(float opacity, float a, float b, float c) {
  const float t = fminf(40.0f, 2.0f * __logf(255.0f * opacity)) * 1.002f + 0.02f;
  const float det = a * c - b * b;
  const float kappa = (a * c) / det;
  float hx = sqrtf(fmaxf(t, 0.0f) * a) * 1.002f + 0.02f;
  float hy = sqrtf(fmaxf(t, 0.0f) * c) * 1.002f + 0.02f;
  if (!(kappa >= 0.0f && kappa <= 64.0f) || !(hx < 60000.0f) || !(hy < 60000.0f)) {
    hx = __int_as_float(0x7f800000);
    hy = __int_as_float(0x7f800000);
  }
  const __half2 h = __halves2half2(__float2half_ru(hx), __float2half_ru(hy));
  return *reinterpret_cast<const uint32_t*>(&h);
}

// True when no Gaussian of a chunk can pass the screen cull of
// project_gaussian for this camera, so the chunk need not be projected.
// With p = R m + t (camera space), u = fx px / pz + cx: the x-row of the
// Jacobian has squared norm (fx/pz)^2 (1 + clamp(px/pz)^2) <= (fx/pz)^2
// (1 + L^2), the camera-space covariance R S R^T has largest eigenvalue at
// most trace(S) times the bound of R^T R's largest eigenvalue (r_scale2),
// and the extent factor is at most sigma, so the pixel radius is below
// bx = 1.01 sigma sqrt((fx/pz)^2 (1 + L^2) tr + eps) + 2 (margins for
// rounding and the ceiling) with tr <= T (the chunk's largest trace times
// r_scale2).  A Gaussian is therefore culled when pz is outside [near, far]
// or u + bx <= 0 (and likewise for the other three image sides).  Since
// sqrt(a + b) <= sqrt(a) + sqrt(b), pz bx / fx <= K + pz m with
// K = 1.01 sigma sqrt((1 + L^2) T) and m = (1.01 sigma sqrt(eps) + 2) / fx,
// and u + bx = (fx / pz)(px + pz cx / fx + pz bx / fx), a Gaussian with
// pz >= near is rejected on the left side whenever
// px + pz (cx / fx + m) + K <= 0: a linear bound in p, whose maximum over
// the chunk's box of means is the value at the centre plus sum |(R^T a)_i|
// h_i.  Every comparison has a relative slack of 1e-4 for rounding, and a
// non-finite bound culls nothing.
__device__ __forceinline__ bool chunk_outside_frustum(const CamConst& c, float4 b0, float4 b1,
                                                      float near_plane, float far_plane,
                                                      float sigma, float eps) {
  if (!(c.fx > 0.0f && c.fy > 0.0f)) return false;
  const float hx = 0.5f * (b1.x - b0.x), hy = 0.5f * (b1.y - b0.y), hz = 0.5f * (b1.z - b0.z);
  const float mx = 0.5f * (b0.x + b1.x), my = 0.5f * (b0.y + b1.y), mz = 0.5f * (b0.z + b1.z);
  const float* R = c.r;
  const float pcx = R[0] * mx + R[1] * my + R[2] * mz + c.t[0];
  const float pcy = R[3] * mx + R[4] * my + R[5] * mz + c.t[1];
  const float pcz = R[6] * mx + R[7] * my + R[8] * mz + c.t[2];
  // sum_i |(R^T a)_i| h_i for the functional a . p.
  auto extent = [&](float a0, float a1, float a2) {
    return fabsf(a0 * R[0] + a1 * R[3] + a2 * R[6]) * hx + fabsf(a0 * R[1] + a1 * R[4] + a2 * R[7]) * hy +
           fabsf(a0 * R[2] + a1 * R[5] + a2 * R[8]) * hz;
  };
  const float ez = extent(0.0f, 0.0f, 1.0f);
  const float sz = 1.0e-4f * (fabsf(pcz) + ez) + 1.0e-6f;
  if (pcz + ez < near_plane - sz) return true;
  if (pcz - ez > far_plane + sz) return true;
  const float t2 = b0.w * c.r_scale2;
  const float lx = fmaxf(c.lim_xp, c.lim_xn), ly = fmaxf(c.lim_yp, c.lim_yn);
  const float kx = 1.01f * sigma * sqrtf((1.0f + lx * lx) * t2) * 1.001f;
  const float ky = 1.01f * sigma * sqrtf((1.0f + ly * ly) * t2) * 1.001f;
  const float m_x = (1.01f * sigma * sqrtf(eps) + 2.0f) / c.fx * 1.001f;
  const float m_y = (1.01f * sigma * sqrtf(eps) + 2.0f) / c.fy * 1.001f;
  // Side planes: low side needs a.p + k > 0 somewhere, high side a.p - k < 0.
  auto low_out = [&](float pc, float az, float ex, float k) {
    const float v = pc + az * pcz + ex + k;
    return v < -(1.0e-4f * (fabsf(pc) + fabsf(az * pcz) + ex + k) + 1.0e-6f);
  };
  auto high_out = [&](float pc, float az, float ex, float k) {
    const float v = pc - az * pcz - ex - k;
    return v > 1.0e-4f * (fabsf(pc) + fabsf(az * pcz) + ex + k) + 1.0e-6f;
  };
  const float ax_lo = c.cx / c.fx + m_x, ax_hi = (c.width - c.cx) / c.fx + m_x;
  const float ay_lo = c.cy / c.fy + m_y, ay_hi = (c.height - c.cy) / c.fy + m_y;
  if (low_out(pcx, ax_lo, extent(1.0f, 0.0f, ax_lo), kx)) return true;
  if (high_out(pcx, ax_hi, extent(1.0f, 0.0f, -ax_hi), kx)) return true;
  if (low_out(pcy, ay_lo, extent(0.0f, 1.0f, ay_lo), ky)) return true;
  if (high_out(pcy, ay_hi, extent(0.0f, 1.0f, -ay_hi), ky)) return true;
  return false;
}

// ---------------------------------------------------------------------------
// Dense mode: optical-thickness depth cutoff (renderer_cuda.cu:247-258,
// 1093-1300, 1658-1689, restructured per tile).  The compositor stops a pixel
// once its transmittance reaches 1e-4, i.e. once sum(-ln(1 - alpha)) >= ln 1e4.
// Pass 1 adds, for every (record, tile) of the cover, a lower bound of the
// record's optical thickness that holds at every pixel of the tile to the
// tile's depth bucket; a tile's cutoff is the first bucket where the bound
// reaches ln 1e4, and pass 2 emits no key behind it.  Every pixel of the tile
// has terminated before the first culled record, so the images are those of
// the plain path, bit for bit.
// ---------------------------------------------------------------------------

// 0.999 * sum_{k=1..8} a^k / k, a lower bound of -ln(1 - a) (the series of
// -ln(1 - a) has positive terms; the factor absorbs float rounding).
__device__ __forceinline__ float conservative_tau(float a) {
  float term = a, sum = a;
#pragma unroll
  for (int k = 2; k <= 8; ++k) {
    term *= a;
    sum += term * (1.0f / static_cast<float>(k));
  }
  return sum * 0.999f;
}

// Lower bound of the compositor's alpha over the pixel centres [x0, x1] x
// [y0, y1]: the conic's quadratic form is convex, so its maximum over the box
// is at a corner; a relative and absolute margin covers the compositor's own
// rounding of q and exp.  0 when some pixel may fall below 1/255 or past the
// power >= -20 cut.
__device__ __forceinline__ float tile_alpha_lower_bound(float mx, float my, float c0, float c1,
                                                        float c2, float o, float x0, float x1,
                                                        float y0, float y1) {
  float qmax = 0.0f;
#pragma unroll
  for (int corner = 0; corner < 4; ++corner) {
    const float dx = ((corner & 1) ? x1 : x0) - mx;
    const float dy = ((corner & 2) ? y1 : y0) - my;
    const float t0 = c0 * dx * dx, t1 = 2.0f * c1 * dx * dy, t2 = c2 * dy * dy;
    const float q = t0 + t1 + t2 + 1.0e-5f * (fabsf(t0) + fabsf(t1) + fabsf(t2)) + 1.0e-4f;
    qmax = fmaxf(qmax, q);
  }
  const float power = -0.5f * qmax;
  if (!(power >= -20.0f)) return 0.0f;
  const float a = fminf(kMaxAlpha, o * vexp(power) * 0.99999f);
  return a >= kAlphaThreshold * 1.0001f ? a : 0.0f;
}

// kRay: exact-ray records (renderer_cuda.cu:795-948) - no early or chunk
// frustum cull (the ellipse cull decides), and each record's precision terms
// go to the extension records p.ray_ext[3 r .. 3 r + 2].
// kMode (ProjectMode): plain fused projection + emission, or one of the two
// dense-mode passes.
template <int kShDegree, bool kRay, int kMode>
__global__ void __launch_bounds__(kProjectThreads, 4) project_emit_kernel(ProjectParams p) {
  __shared__ Record s_rec[kProjectChunk];          // by task slot
  __shared__ uint16_t s_slot[kProjectChunk];       // rank -> task slot
  // By task slot, like s_rec (held in shared memory rather than registers
  // across the two projection rounds).
  __shared__ uint32_t s_rect_min[kProjectChunk];   // min_tx | min_ty << 16
  __shared__ uint32_t s_rect_size[kProjectChunk];  // ntx | nty << 16
  __shared__ uint32_t s_prefix[kProjectChunk + 1]; // exclusive isect prefix
  __shared__ uint16_t s_owner[kOwnerKeys];         // key -> record rank (blocks of <= kOwnerKeys keys)
  __shared__ int32_t s_radii[kProjectChunk * 2];
  __shared__ uint32_t s_warp_vis[kProjectRounds][kProjectThreads / 32];
  __shared__ uint64_t s_warp_isect[kProjectRounds][kProjectThreads / 32];
  __shared__ CamConst s_cams[kTicketBatch];
  __shared__ __align__(8) CamPlan s_plans[kTicketBatch];
  __shared__ int64_t s_vbs[kTicketBatch];
  __shared__ uint32_t s_cmask[kTicketBatch];  // live clusters of each staged block
  __shared__ int s_nlive;
  __shared__ int s_exhausted;
  __shared__ uint64_t s_base_vis, s_base_isect;
  __shared__ uint32_t s_nvis;
  __shared__ uint32_t s_nisect;

  ScratchHeader* header = reinterpret_cast<ScratchHeader*>(p.scratch + p.layout.header);
  const CamPlan* plans = reinterpret_cast<const CamPlan*>(p.scratch + p.layout.plans);
  const CamConst* cam_consts = reinterpret_cast<const CamConst*>(p.scratch + p.layout.cam_consts);
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;

  const int64_t total_vblocks = p.total_vblocks;
  int cursor = 0;
  int nlive = 0;
  while (true) {
    if (cursor == nlive) {
      // Warp 0 takes kTicketBatch consecutive virtual blocks; each lane
      // stages one (plan, projection constants) and drops it when it adds
      // nothing (an invalid camera, a chunk past its camera's scene, a chunk
      // outside the frustum); the rest are compacted into shared memory.
      // The previous vblock ended with a barrier, so the arrays are free.
      if (warp == 0) {
        int64_t base = 0;
        if (lane == 0) base = atomicAdd(&header->project_queue, static_cast<uint32_t>(kTicketBatch));
        base = __shfl_sync(0xffffffffu, base, 0);
        const int64_t vb = base + lane;
        bool live = vb < total_vblocks;
        const int64_t slot = live ? vb % p.active_count : 0;
        if (live) {
          const int64_t chunk = vb / p.active_count;
          const CamPlan& plan = plans[slot];
          const int scene_slot = plan.scene_slot;
          live = plan.camera >= 0 && scene_slot >= 0 && chunk * kProjectChunk < plan.g_count;
          if (live && p.chunk_bounds && !kRay) {
            const int64_t ci = p.chunk_offsets[scene_slot] + chunk;
            live = !chunk_outside_frustum(cam_consts[slot], p.chunk_bounds[ci * 2],
                                          p.chunk_bounds[ci * 2 + 1], p.near_plane, p.far_plane,
                                          p.support_sigma, p.cov_eps);
          }
        }
        const uint32_t mask = __ballot_sync(0xffffffffu, live);
        if (live) {
          const int rank = __popc(mask & ((1u << lane) - 1u));
#pragma unroll
          for (int w = 0; w < 7; ++w) {
            reinterpret_cast<uint64_t*>(&s_plans[rank])[w] =
                reinterpret_cast<const uint64_t*>(plans + slot)[w];
          }
#pragma unroll
          for (int w = 0; w < 7; ++w) {
            reinterpret_cast<float4*>(&s_cams[rank])[w] = reinterpret_cast<const float4*>(cam_consts + slot)[w];
          }
          s_vbs[rank] = vb;
        }
        if (lane == 0) {
          s_nlive = __popc(mask);
          s_exhausted = base + kTicketBatch >= total_vblocks;
        }
      }
      __syncthreads();
      nlive = s_nlive;
      cursor = 0;
      if (nlive == 0) {
        if (s_exhausted) break;
        continue;
      }
      if (p.cluster_bounds && !kRay) {
        // Cluster cull of the staged blocks, the chunk test on each
        // cluster's box: bit k of s_cmask[v] is set when cluster k (tasks
        // [32 k, 32 k + 32) of block v, one warp-round) may hold a Gaussian
        // the screen cull keeps.  One lane per cluster; 32 lanes cover two
        // blocks.
        static_assert(kProjectClusters == 16, "two blocks' clusters per warp ballot");
        for (int base = warp * 32; base < nlive * kProjectClusters; base += kProjectThreads) {
          const int idx = base + lane;
          bool keep = true;
          if (idx < nlive * kProjectClusters) {
            const int v = idx / kProjectClusters;
            const int64_t ci = p.chunk_offsets[s_plans[v].scene_slot] + s_vbs[v] / p.active_count;
            const int64_t row = ci * kProjectClusters + (idx - v * kProjectClusters);
            keep = !chunk_outside_frustum(s_cams[v], p.cluster_bounds[row * 2], p.cluster_bounds[row * 2 + 1],
                                          p.near_plane, p.far_plane, p.support_sigma, p.cov_eps);
          }
          const uint32_t bits = __ballot_sync(0xffffffffu, keep);
          const int v0 = base / kProjectClusters;
          if (lane == 0) s_cmask[v0] = bits & 0xffffu;
          if (lane == 16 && v0 + 1 < nlive) s_cmask[v0 + 1] = bits >> 16;
        }
        __syncthreads();
      }
    }
    const int64_t b = s_vbs[cursor];
    const CamPlan& plan = s_plans[cursor];
    const CamConst& s_cam = s_cams[cursor];
    const uint32_t cluster_mask = p.cluster_bounds && !kRay ? s_cmask[cursor] : 0xffffffffu;
    ++cursor;
    const int64_t chunk = b / p.active_count;
    const int64_t local_begin = chunk * kProjectChunk;
    const bool live = true;

    // Project both rounds first (no barrier), then one block scan of
    // (visible, tiles) over the kProjectChunk tasks in task order.
    bool vis[kProjectRounds];
    uint32_t ntiles[kProjectRounds];
    float ray_terms[kRay ? kProjectRounds : 1][10];
    uint32_t ray_rank[kRay ? kProjectRounds : 1];
    const float its = 1.0f / static_cast<float>(p.tile_size);
#pragma unroll
    for (int round = 0; round < kProjectRounds; ++round) {
      const int64_t local = local_begin + round * kProjectThreads + tid;
      vis[round] = false;
      ntiles[round] = 0;
      Projected pr;
      if (live && local < plan.g_count && ((cluster_mask >> (round * (kProjectThreads / 32) + warp)) & 1u)) {
        const int64_t g = plan.g_begin + local;
        vis[round] = project_gaussian<kRay>(p.means, p.covariances, p.opacities, g, s_cam, p.near_plane,
                                      p.far_plane, p.support_sigma, p.cov_eps, p.antialiased, &pr);
        if (vis[round]) {
          const float frx = static_cast<float>(pr.radius_x);
          const float fry = static_cast<float>(pr.radius_y);
          const int min_tx = max(0, floor_clamped(fsub(fmul(pr.mean_x, its), fmul(frx, its))));
          const int min_ty = max(0, floor_clamped(fsub(fmul(pr.mean_y, its), fmul(fry, its))));
          const int max_tx =
              min(plan.tiles_x, ceil_clamped(fadd(fmul(pr.mean_x, its), fmul(frx, its))));
          const int max_ty =
              min(plan.tiles_y, ceil_clamped(fadd(fmul(pr.mean_y, its), fmul(fry, its))));
          const int ntx = max(0, max_tx - min_tx);
          const int nty = max(0, max_ty - min_ty);
          ntiles[round] = static_cast<uint32_t>(ntx) * static_cast<uint32_t>(nty);
          if (kMode == kProjectDenseTau) {
            // Pass 1: optical-thickness lower bounds into the record's depth
            // bucket of the kDenseSubtile cells inside its core, the box of
            // the ellipse where alpha >= kDenseMinAlpha; nothing is emitted.
            // Leaving the fainter rim out only lowers the bounds.
            const int bucket = dense_bucket(pr.depth, p.near_bits);
            const float qc = 2.0f * __logf(pr.opacity * (1.0f / kDenseMinAlpha));
            const int64_t sub_base = static_cast<int64_t>(plan.camera) * p.sub_x * p.sub_y;
            constexpr float kCell = static_cast<float>(kDenseSubtile);
            const float hx = qc > 0.0f ? sqrtf(qc * pr.cov_a) : -1.0f;
            const float hy = qc > 0.0f ? sqrtf(qc * pr.cov_c) : -1.0f;
            // Cells whose pixel centres [4s + 0.5, 4s + 3.5] lie in the box.
            const int sx0 = max(0, ceil_clamped((pr.mean_x - hx - 0.5f) * (1.0f / kCell)));
            const int sx1 = min(p.sub_x - 1, floor_clamped((pr.mean_x + hx - 3.5f) * (1.0f / kCell)));
            const int sy0 = max(0, ceil_clamped((pr.mean_y - hy - 0.5f) * (1.0f / kCell)));
            const int sy1 = min(p.sub_y - 1, floor_clamped((pr.mean_y + hy - 3.5f) * (1.0f / kCell)));
            for (int sy = sy0; hy >= 0.0f && sy <= sy1; ++sy) {
              const float y0 = static_cast<float>(sy) * kCell + 0.5f;
              const float y1 = fminf(y0 + kCell - 1.0f, static_cast<float>(plan.height) - 0.5f);
              for (int sx = sx0; sx <= sx1; ++sx) {
                const float x0 = static_cast<float>(sx) * kCell + 0.5f;
                const float x1 = fminf(x0 + kCell - 1.0f, static_cast<float>(plan.width) - 0.5f);
                const float a = tile_alpha_lower_bound(pr.mean_x, pr.mean_y, pr.conic0, pr.conic1,
                                                       pr.conic2, pr.opacity, x0, x1, y0, y1);
                if (a > 0.0f) {
                  const int64_t cell = sub_base + static_cast<int64_t>(sy) * p.sub_x + sx;
                  atomicAdd(p.depth_tau + cell * kDenseBuckets + bucket, conservative_tau(a));
                }
              }
            }
            vis[round] = false;
            ntiles[round] = 0;
          } else if (kMode == kProjectDenseCull) {
            // Pass 2: only the tiles whose cutoff bucket is not in front of
            // the record; a record left with none is not emitted.
            const int bucket = dense_bucket(pr.depth, p.near_bits);
            uint32_t kept = 0;
            for (int ty = min_ty; ty < min_ty + nty; ++ty) {
              const int64_t row = plan.tile_base + static_cast<int64_t>(ty) * plan.tiles_x;
              for (int tx = min_tx; tx < min_tx + ntx; ++tx) kept += bucket <= p.tile_cutoff[row + tx];
            }
            ntiles[round] = kept;
            if (kept == 0) vis[round] = false;
          }
        }
        if (vis[round]) {
          const float frx = static_cast<float>(pr.radius_x);
          const float fry = static_cast<float>(pr.radius_y);
          const int min_tx = max(0, floor_clamped(fsub(fmul(pr.mean_x, its), fmul(frx, its))));
          const int min_ty = max(0, floor_clamped(fsub(fmul(pr.mean_y, its), fmul(fry, its))));
          const int ntx = max(0, min(plan.tiles_x, ceil_clamped(fadd(fmul(pr.mean_x, its), fmul(frx, its)))) - min_tx);
          const int nty = max(0, min(plan.tiles_y, ceil_clamped(fadd(fmul(pr.mean_y, its), fmul(fry, its)))) - min_ty);
          const int slot = round * kProjectThreads + tid;
          s_rect_min[slot] = static_cast<uint32_t>(min(min_tx, 65535)) |
                             (static_cast<uint32_t>(min(min_ty, 65535)) << 16);
          s_rect_size[slot] = static_cast<uint32_t>(ntx) | (static_cast<uint32_t>(nty) << 16);
          s_radii[slot * 2 + 0] = pr.radius_x;
          s_radii[slot * 2 + 1] = pr.radius_y;
          if (kRay) {
#pragma unroll
            for (int k = 0; k < 6; ++k) ray_terms[kRay ? round : 0][k] = pr.prec[k];
#pragma unroll
            for (int k = 0; k < 3; ++k) ray_terms[kRay ? round : 0][6 + k] = pr.prec_mean[k];
            ray_terms[kRay ? round : 0][9] = pr.mean_prec_mean;
          }
          // Staged by task slot; the scan below maps ranks to slots.  The
          // colour is evaluated after the scan, over the compacted visible
          // records (full warps), from the camera-space position kept in
          // c.x / c.y (c.z unused until then; z is the depth b.z).
          Record& staged = s_rec[round * kProjectThreads + tid];
          staged.a = make_float4(pr.mean_x, pr.mean_y, pr.conic0, pr.conic1);
          const int32_t id = p.gaussian_ids ? p.gaussian_ids[g] : static_cast<int32_t>(g);
          staged.b = make_float4(pr.conic2, pr.opacity, pr.depth, __int_as_float(id));
          // c.w: the screen-space alpha footprint, or in exact-ray mode the
          // half-extents (radius + 1 px, 16-bit each, 32767 = unbounded) of
          // the ray ellipse's box around its centre.
          const uint32_t box =
              kRay ? static_cast<uint32_t>(min(pr.radius_x, 32766) + 1) |
                         (static_cast<uint32_t>(min(pr.radius_y, 32766) + 1) << 16)
                   : footprint_box(pr.opacity, pr.cov_a, pr.cov_b, pr.cov_c);
          staged.c = make_float4(pr.px, pr.py, 0.0f, __uint_as_float(box));
        }
      }
    }
    uint32_t v_incl[kProjectRounds];
    uint64_t t_incl[kProjectRounds];
#pragma unroll
    for (int round = 0; round < kProjectRounds; ++round) {
      v_incl[round] = vis[round] ? 1u : 0u;
      t_incl[round] = ntiles[round];
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t nv = __shfl_up_sync(0xffffffffu, v_incl[round], o);
        const uint64_t nt = __shfl_up_sync(0xffffffffu, t_incl[round], o);
        if (lane >= o) {
          v_incl[round] += nv;
          t_incl[round] += nt;
        }
      }
      if (lane == 31) {
        s_warp_vis[round][warp] = v_incl[round];
        s_warp_isect[round][warp] = t_incl[round];
      }
    }
    __syncthreads();
    uint32_t block_vis = 0;
    uint64_t block_isect = 0;
#pragma unroll
    for (int round = 0; round < kProjectRounds; ++round) {
      uint32_t wv = 0, rv = 0;
      uint64_t wt = 0, rt = 0;
#pragma unroll
      for (int w = 0; w < kProjectThreads / 32; ++w) {
        const uint32_t sv = s_warp_vis[round][w];
        const uint64_t st = s_warp_isect[round][w];
        if (w < warp) {
          wv += sv;
          wt += st;
        }
        rv += sv;
        rt += st;
      }
      if (vis[round]) {
        const uint32_t rank = block_vis + wv + v_incl[round] - 1;
        const uint64_t excl = block_isect + wt + t_incl[round] - ntiles[round];
        s_slot[rank] = static_cast<uint16_t>(round * kProjectThreads + tid);
        s_prefix[rank] = static_cast<uint32_t>(excl > 0x7fffffffull ? 0x7fffffffull : excl);
        if (kRay) ray_rank[kRay ? round : 0] = rank;
        // Owner of each of the record's keys, for blocks whose keys fit
        // (the emission below falls back to a search of s_prefix otherwise).
        for (uint64_t k = excl; k < excl + ntiles[round] && k < static_cast<uint64_t>(kOwnerKeys); ++k) {
          s_owner[k] = static_cast<uint16_t>(rank);
        }
      }
      block_vis += rv;
      block_isect += rt;
    }
    if (tid == 0) {
      s_nvis = block_vis;
      s_prefix[block_vis] =
          static_cast<uint32_t>(block_isect > 0x7fffffffull ? 0x7fffffffull : block_isect);
      s_nisect = s_prefix[block_vis];
    }

    // The block's output ranges: one reservation of (visible, intersection)
    // slots per block, no waiting on other blocks.  The order of the blocks'
    // ranges is therefore not fixed, but within a block records and keys stay
    // in task order, and the tile sort orders every tile by (depth bits,
    // Gaussian id), which does not depend on where the records landed.
    if (tid == 0) {
      s_base_vis = atomicAdd(&header->visible_total, static_cast<unsigned long long>(block_vis));
      s_base_isect = atomicAdd(&header->isect_total, static_cast<unsigned long long>(block_isect));
    }
    __syncthreads();

    const uint32_t nvis = s_nvis;
    if (nvis > 0) {
      const uint64_t base_vis = s_base_vis;
      const uint64_t base_isect = s_base_isect;
      const uint64_t vcap = static_cast<uint64_t>(p.visible_capacity);
      const uint64_t icap = static_cast<uint64_t>(p.intersection_capacity);
      // Records in rank order, one thread per record: the colour (SH or
      // linear RGB) of the record's Gaussian, then the three float4s.
      float4* dst = reinterpret_cast<float4*>(p.records);
      for (uint32_t i = tid; i < nvis; i += kProjectThreads) {
        const uint32_t slot = s_slot[i];
        const Record& st = s_rec[slot];
        const int64_t g = plan.g_begin + local_begin + slot;
        float rgb[3];
        if (kShDegree < 0) {
          rgb[0] = p.features[g * p.feature_width + 0];
          rgb[1] = p.features[g * p.feature_width + 1];
          rgb[2] = p.features[g * p.feature_width + 2];
        } else {
          eval_sh<kShDegree < 0 ? 0 : kShDegree>(p.features + g * p.feature_width, p.wide_feature_loads,
                                                 p.vector_feature_loads, s_cam, st.c.x, st.c.y, st.b.z, rgb);
        }
        const uint64_t r = base_vis + i;
        if (r < vcap) {
          dst[r * 3 + 0] = st.a;
          dst[r * 3 + 1] = st.b;
          dst[r * 3 + 2] = make_float4(rgb[0], rgb[1], rgb[2], st.c.w);
        }
      }
      if (kRay) {
        // Extension records: each thread writes its own visible Gaussians'.
#pragma unroll
        for (int round = 0; round < kProjectRounds; ++round) {
          const uint64_t r = base_vis + ray_rank[kRay ? round : 0];
          if (vis[round] && r < vcap) {
            const float* t = ray_terms[kRay ? round : 0];
            p.ray_ext[r * 3 + 0] = make_float4(t[0], t[1], t[2], t[3]);
            p.ray_ext[r * 3 + 1] = make_float4(t[4], t[5], t[6], t[7]);
            p.ray_ext[r * 3 + 2] = make_float4(t[8], t[9], 0.0f, 0.0f);
            if (p.mirror_ray_precisions) {
              // Reference workspace layout (renderer_cuda.cu:1056-1071).
#pragma unroll
              for (int k = 0; k < 6; ++k) p.mirror_ray_precisions[r * 6 + k] = t[k];
#pragma unroll
              for (int k = 0; k < 4; ++k) p.mirror_ray_precision_means[r * 4 + k] = t[6 + k];
            }
          }
        }
      }
      if (p.record_map) {
        // Training: record index of each visible (slot, Gaussian), for the
        // per-Gaussian backward pass.
        int32_t* map_row = p.record_map + (b % p.active_count) * p.record_map_stride;
        for (uint32_t i = tid; i < nvis; i += kProjectThreads) {
          const uint64_t r = base_vis + i;
          const int64_t local = local_begin + s_slot[i];
          if (r < vcap) map_row[local] = static_cast<int32_t>(r);
        }
      }
      if (p.mirror_means2d) {
        for (uint32_t i = tid; i < nvis; i += kProjectThreads) {
          const uint64_t r = base_vis + i;
          if (r >= vcap) continue;
          const Record rec = s_rec[s_slot[i]];
          p.mirror_means2d[r * 2 + 0] = rec.a.x;
          p.mirror_means2d[r * 2 + 1] = rec.a.y;
          p.mirror_conics[r * 3 + 0] = rec.a.z;
          p.mirror_conics[r * 3 + 1] = rec.a.w;
          p.mirror_conics[r * 3 + 2] = rec.b.x;
          p.mirror_depths[r] = rec.b.z;
          p.mirror_opacities[r] = rec.b.y;
          p.mirror_camera_ids[r] = plan.camera;
          p.mirror_gaussian_ids[r] = __float_as_int(rec.b.w);
          p.mirror_radii[r * 2 + 0] = s_radii[s_slot[i] * 2 + 0];
          p.mirror_radii[r * 2 + 1] = s_radii[s_slot[i] * 2 + 1];
        }
      }
      // Tile intersections: one key per covered tile, cooperative over the
      // block's prefix so consecutive threads store consecutive keys.
      const uint32_t nisect = s_nisect;
      uint64_t limit = 0;
      if (base_isect < icap) {
        const uint64_t room = icap - base_isect;
        limit = room < nisect ? room : nisect;
      }
      const int64_t tiles_x = plan.tiles_x;
      if (kMode == kProjectDenseCull) {
        // Dense mode: each record's kept tiles in rect order, one thread per
        // record (the kept tiles are not a dense range of the rect).
        for (uint32_t i = tid; i < nvis; i += kProjectThreads) {
          const uint64_t r = base_vis + i;
          const uint32_t slot = s_slot[i];
          const float depth = s_rec[slot].b.z;
          const int bucket = dense_bucket(depth, p.near_bits);
          const uint32_t ntx = s_rect_size[slot] & 0xffffu;
          const uint32_t nty = s_rect_size[slot] >> 16;
          const uint32_t min_tx = s_rect_min[slot] & 0xffffu;
          const uint32_t min_ty = s_rect_min[slot] >> 16;
          uint32_t j = s_prefix[i];
          for (uint32_t ty = min_ty; ty < min_ty + nty; ++ty) {
            for (uint32_t tx = min_tx; tx < min_tx + ntx; ++tx) {
              const uint64_t tile = static_cast<uint64_t>(plan.tile_base) + static_cast<uint64_t>(ty) * tiles_x + tx;
              if (bucket > p.tile_cutoff[tile]) continue;
              if (j < limit) {
                uint64_t key = ~0ull;
                int32_t value = 0;
                if (r < vcap) {
                  key = (tile << 32) | static_cast<uint64_t>(__float_as_uint(depth));
                  value = static_cast<int32_t>(r);
                  if (tile < static_cast<uint64_t>(p.tile_count)) atomicAdd(p.tile_counts + tile, 1u);
                }
                p.keys[base_isect + j] = key;
                p.values[base_isect + j] = value;
              }
              ++j;
            }
          }
        }
      }
      const bool owner_table = nisect <= static_cast<uint32_t>(kOwnerKeys);
      for (uint32_t j = tid; j < limit && kMode != kProjectDenseCull; j += kProjectThreads) {
        // Owner record: last i with s_prefix[i] <= j.
        uint32_t i;
        if (owner_table) {
          i = s_owner[j];
        } else {
          uint32_t lo = 0, hi = nvis;  // invariant s_prefix[lo] <= j < s_prefix[hi]
          while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (s_prefix[mid] <= j) lo = mid; else hi = mid;
          }
          i = lo;
        }
        const uint32_t local = j - s_prefix[i];
        const uint32_t slot = s_slot[i];
        const uint32_t ntx = s_rect_size[slot] & 0xffffu;
        const uint32_t ty = ntx == 1u ? local : local / ntx;  // most records span one tile column
        const uint32_t tx = local - ty * ntx;
        const uint32_t min_tx = s_rect_min[slot] & 0xffffu;
        const uint32_t min_ty = s_rect_min[slot] >> 16;
        const uint64_t r = base_vis + i;
        uint64_t key = ~0ull;
        int32_t value = 0;
        const uint64_t tile = static_cast<uint64_t>(plan.tile_base) +
                              static_cast<uint64_t>(min_ty + ty) * tiles_x + (min_tx + tx);
        if (r < vcap) {
          key = (tile << 32) | static_cast<uint64_t>(__float_as_uint(s_rec[slot].b.z));
          value = static_cast<int32_t>(r);
        }
        // Bucket size for the tile sort (a tile past the batch's range - a
        // caller's inconsistent ragged offsets - is left to the scatter's
        // overflow tail): one atomic per group of lanes with the same tile.
        const bool counted = r < vcap && tile < static_cast<uint64_t>(p.tile_count);
        const unsigned active = __activemask();
        const unsigned peers = __match_any_sync(active, counted ? static_cast<uint32_t>(tile) : 0xffffffffu);
        if (counted && (threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(p.tile_counts + tile, __popc(peers));
        p.keys[base_isect + j] = key;
        p.values[base_isect + j] = value;
      }
    }
    __syncthreads();
  }
}

#define VGR_PROJECT_VARIANTS(RAY, MODE)                                   \
  template __global__ void project_emit_kernel<-1, RAY, MODE>(ProjectParams); \
  template __global__ void project_emit_kernel<0, RAY, MODE>(ProjectParams);  \
  template __global__ void project_emit_kernel<1, RAY, MODE>(ProjectParams);  \
  template __global__ void project_emit_kernel<2, RAY, MODE>(ProjectParams);  \
  template __global__ void project_emit_kernel<3, RAY, MODE>(ProjectParams);
VGR_PROJECT_VARIANTS(false, kProjectPlain)
VGR_PROJECT_VARIANTS(true, kProjectPlain)
VGR_PROJECT_VARIANTS(false, kProjectDenseTau)
VGR_PROJECT_VARIANTS(false, kProjectDenseCull)
#undef VGR_PROJECT_VARIANTS

// Depth cutoff (renderer_cuda.cu:1658-1689): one warp per cell scans its
// kDenseBuckets optical-thickness bounds (8 per lane) for the first bucket
// where the running sum reaches ln 1e4 (the compositor's T <= 1e-4 stop), or
// the last bucket; a tile's cutoff is the largest of its cells'.  Thread 0
// of block 0 also rewinds the projection ticket for the second pass.
__global__ void __launch_bounds__(256) dense_cutoff_kernel(DenseCutoffParams p) {
  constexpr float kStopTau = 9.210340371976184f;  // ln(1e4)
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    reinterpret_cast<ScratchHeader*>(p.scratch + p.layout.header)->project_queue = 0u;
  }
  const int lane = threadIdx.x & 31;
  const int64_t cell = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  if (cell >= p.sub_count) return;
  const float4* row = reinterpret_cast<const float4*>(p.depth_tau + cell * kDenseBuckets) + lane * 2;
  const float4 a = row[0], b = row[1];
  const float v[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
  float local = 0.0f;
#pragma unroll
  for (int k = 0; k < 8; ++k) local += v[k];
  float incl = local;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const float n = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += n;
  }
  int first = kDenseBuckets;
  if (incl >= kStopTau) {
    float run = incl - local;
    for (int k = 0; k < 8; ++k) {
      run += v[k];
      if (run >= kStopTau) {
        first = lane * 8 + k;
        break;
      }
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) first = min(first, __shfl_xor_sync(0xffffffffu, first, o));
  if (lane == 0) {
    const int64_t per_image = static_cast<int64_t>(p.sub_x) * p.sub_y;
    const int64_t image = cell / per_image;
    const int64_t local = cell - image * per_image;
    const int sy = static_cast<int>(local / p.sub_x);
    const int sx = static_cast<int>(local - static_cast<int64_t>(sy) * p.sub_x);
    const int per_tile = p.tile_size / kDenseSubtile;
    const int64_t tile = image * p.tiles_per_image + static_cast<int64_t>(sy / per_tile) * p.tiles_x + sx / per_tile;
    atomicMax(p.tile_cutoff + tile, first < kDenseBuckets ? first : kDenseBuckets - 1);
  }
}

}  // namespace vgr
