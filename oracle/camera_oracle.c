/*
 * camera_oracle.c -- CPU restatement of the reference camera path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity oracle of the camera
 * renderer: tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg
 * load it (as liboracle_camera.so) to check or time the CUDA path; nothing in
 * the product imports, links or executes it.
 *
 * It follows the reference equation of
 *   src/isaacsim_gaussian_renderer/native/renderer_cuda.cu
 *     :112-143   quaternion -> rotation
 *     :492-540   object covariance R S S^T R^T
 *     :287-490   EWA projection, near/far cull, 1.3x FOV clamp, +eps
 *                dilation, Mip-Splatting compensation, radius, screen cull,
 *                conic
 *     :1691-1829 tile cover [floor(m/ts - r/ts), ceil(m/ts + r/ts)) and key
 *     :1944-1971 deterministic order (tile, depth bits, Gaussian id)
 *     :1973-2305 front-to-back compositor (RGB, alpha, depth, semantic)
 *     :161-166   sRGB transfer
 *     :795-948   exact-ray mode: FP64 camera-space precision, ray-ellipse
 *                cull centre and radius
 *     :203-245, 2190-2270  exact-ray alpha and blend-then-stop compositing
 * with every floating-point operation written in a fixed order with
 * contraction disabled (built with -ffp-contract=off; fmaf only where a fused
 * multiply-add is intended), and exp/log evaluated by the Cody-Waite/minimax
 * and atanh-series methods spelled out below.  The CUDA kernels perform the
 * identical operation sequence, so outputs agree bit for bit.  Against the
 * reference's own CUDA build (compiled with --use_fast_math, __expf/__logf)
 * results agree within the stated float tolerances instead.
 *
 * Spherical harmonics (sh_degree >= 0) have no counterpart in the reference,
 * which reads features[0..2] as linear RGB (sh_degree = -1): they follow the
 * real-SH basis of the 3D Gaussian Splatting reference implementation as used
 * by gsplat (parity unpinned by any reference fixture).
 */
#include <limits.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

#define ALPHA_THRESHOLD (1.0f / 255.0f)
#define MAX_ALPHA 0.99f
#define TRANSMITTANCE_THRESHOLD 1.0e-4f
#define MIN_AA_COMPENSATION 0.005f

typedef struct vo_scene {
  const float* means;
  const float* covariances;
  const float* opacities;
  const float* features;
  int64_t feature_width;
  const int64_t* semantic_ids;
  const int64_t* registered_scene_ids;
  const int64_t* scene_offsets;
  int64_t scene_count;
} vo_scene;

typedef struct vo_cameras {
  const float* viewmats;
  const float* intrinsics;
  const float* env_xforms;
  const int64_t* camera_scene_ids;
  const int64_t* active_ids; /* NULL: all cameras */
  int64_t batch;
  int64_t active_count;
  const int32_t* widths; /* ragged form or NULL */
  const int32_t* heights;
  const int64_t* tile_offsets;
  const int64_t* pixel_offsets;
} vo_cameras;

typedef struct vo_options {
  int64_t height;
  int64_t width;
  double near_plane;
  double far_plane;
  double support_sigma;
  double covariance_epsilon;
  double semantic_min_alpha;
  int32_t antialiased;
  int32_t tile_size;
  int32_t output_srgb;
  int32_t full_sensor_output;
  int32_t sh_degree;
  int32_t threads;
  int32_t ray_eval; /* exact ray-Gaussian evaluation (renderer_cuda.cu:203-245,795-948) */
} vo_options;

typedef struct vo_stats {
  int64_t visible;
  int64_t intersections;
  int64_t active_tiles;
} vo_stats;

static float bits_to_float(uint32_t u) {
  float f;
  memcpy(&f, &u, 4);
  return f;
}
static uint32_t float_to_bits(float f) {
  uint32_t u;
  memcpy(&u, &f, 4);
  return u;
}

/* exp(x): x log2 e = n + f, n = rint, f by two fma steps against a split
 * log2 e, 2^f by the degree-5 minimax polynomial on |f| <= 1/2 (relative
 * error 7.5e-8, coefficients rounded to float; the same method and constants
 * as the CUDA kernels' vexp), times 2^n built in the exponent field. */
static float vo_exp(float x) {
  const float log2e_hi = 1.44269502162933349609375f;
  const float log2e_lo = 1.925963033500011079e-8f;
  const float t = x * log2e_hi;
  const float n = rintf(t);
  float f = fmaf(x, log2e_hi, -n);
  f = fmaf(x, log2e_lo, f);
  float p = 1.327647245e-03f; /* degree-5 minimax of 2^f on |f| <= 1/2 */
  p = fmaf(p, f, 9.675540961e-03f);
  p = fmaf(p, f, 5.550713092e-02f);
  p = fmaf(p, f, 2.402212024e-01f);
  p = fmaf(p, f, 6.931469440e-01f);
  p = fmaf(p, f, 1.000000119e+00f);
  const int e = (int)n;
  return p * bits_to_float((uint32_t)(e + 127) << 23);
}

/* ln(y): y = m 2^e, m folded into [sqrt(1/2), sqrt(2)), ln m = 2 atanh(s) with
 * s = (m-1)/(m+1) and the odd series through s^11, plus e ln 2 (split). */
static float vo_log(float y) {
  const uint32_t bits = float_to_bits(y);
  int e = (int)((bits >> 23) & 0xffu) - 127;
  float m = bits_to_float((bits & 0x007fffffu) | 0x3f800000u);
  if (m > 1.41421353816986083984375f) {
    m = m * 0.5f;
    e += 1;
  }
  const float s = (m - 1.0f) / (m + 1.0f);
  const float s2 = s * s;
  float p = 0.0909090909090909f;
  p = fmaf(p, s2, 0.1111111111111111f);
  p = fmaf(p, s2, 0.1428571428571428f);
  p = fmaf(p, s2, 0.2f);
  p = fmaf(p, s2, 0.3333333333333333f);
  p = fmaf(p, s2, 1.0f);
  const float lnm = (2.0f * s) * p;
  const float fe = (float)e;
  return fmaf(fe, 0.693145751953125f, fmaf(fe, 1.428606765330187e-06f, lnm));
}

static float vo_srgb(float v) {
  v = fminf(fmaxf(v, 0.0f), 1.0f);
  if (v <= 0.0031308f) return 12.92f * v;
  const float p = vo_exp(vo_log(v) * 0.4166666666666667f);
  return 1.055f * p - 0.055f;
}

/* float -> int with CUDA's conversion semantics (saturating, NaN -> 0);
 * C leaves out-of-range conversions undefined. */
static int saturating_int(float x) {
  if (!(x == x)) return 0;
  if (x >= 2147483648.0f) return INT_MAX;
  if (x <= -2147483648.0f) return INT_MIN;
  return (int)x;
}
static int ceil_radius(float x) {
  return x > 0.0f ? (int)fminf(ceilf(x), 2147483520.0f) : 0;
}
static int floor_clamped(float x) {
  if (!(x == x)) return 0;
  return (int)floorf(fminf(fmaxf(x, -1073741824.0f), 1073741824.0f));
}
static int ceil_clamped(float x) {
  if (!(x == x)) return 0;
  return (int)ceilf(fminf(fmaxf(x, -1073741824.0f), 1073741824.0f));
}

void vo_precompute_covariances(const float* scales, const float* rotations, int64_t count,
                               float* out) {
  for (int64_t g = 0; g < count; ++g) {
    float w = rotations[g * 4 + 0], x = rotations[g * 4 + 1];
    float y = rotations[g * 4 + 2], z = rotations[g * 4 + 3];
    const float norm2 = fmaf(z, z, fmaf(y, y, fmaf(x, x, w * w)));
    const float inv = 1.0f / sqrtf(fmaxf(norm2, 1.0e-20f));
    w = w * inv;
    x = x * inv;
    y = y * inv;
    z = z * inv;
    const float xx = x * x, yy = y * y, zz = z * z;
    const float xy = x * y, xz = x * z, yz = y * z;
    const float wx = w * x, wy = w * y, wz = w * z;
    float r[9];
    r[0] = 1.0f - 2.0f * (yy + zz);
    r[1] = 2.0f * (xy - wz);
    r[2] = 2.0f * (xz + wy);
    r[3] = 2.0f * (xy + wz);
    r[4] = 1.0f - 2.0f * (xx + zz);
    r[5] = 2.0f * (yz - wx);
    r[6] = 2.0f * (xz - wy);
    r[7] = 2.0f * (yz + wx);
    r[8] = 1.0f - 2.0f * (xx + yy);
    const float sx = scales[g * 3 + 0], sy = scales[g * 3 + 1], sz = scales[g * 3 + 2];
    const float s2[3] = {sx * sx, sy * sy, sz * sz};
    static const int rows[6][2] = {{0, 0}, {0, 1}, {0, 2}, {1, 1}, {1, 2}, {2, 2}};
    for (int k = 0; k < 6; ++k) {
      const float* a = r + rows[k][0] * 3;
      const float* b = r + rows[k][1] * 3;
      out[g * 6 + k] = fmaf(a[2] * b[2], s2[2], fmaf(a[1] * b[1], s2[1], (a[0] * b[0]) * s2[0]));
    }
  }
}

typedef struct cam_const {
  float r[9], t[3];
  float fx, fy, cx, cy;
  float lim_xp, lim_xn, lim_yp, lim_yn;
  float width, height;
} cam_const;

static void make_cam_const(const float* view, const float* env, const float* intr, int width,
                           int height, cam_const* c) {
  for (int row = 0; row < 3; ++row) {
    for (int col = 0; col < 3; ++col) {
      c->r[row * 3 + col] = fmaf(view[row * 4 + 2], env[8 + col],
                                 fmaf(view[row * 4 + 1], env[4 + col], view[row * 4 + 0] * env[col]));
    }
    c->t[row] = fmaf(view[row * 4 + 2], env[11],
                     fmaf(view[row * 4 + 1], env[7], fmaf(view[row * 4 + 0], env[3], view[row * 4 + 3])));
  }
  c->fx = intr[0];
  c->fy = intr[4];
  c->cx = intr[2];
  c->cy = intr[5];
  const float w = (float)width, h = (float)height;
  c->width = w;
  c->height = h;
  const float tan_x = (0.5f * w) / c->fx;
  const float tan_y = (0.5f * h) / c->fy;
  c->lim_xp = fmaf(0.3f, tan_x, (w - c->cx) / c->fx);
  c->lim_xn = fmaf(0.3f, tan_x, c->cx / c->fx);
  c->lim_yp = fmaf(0.3f, tan_y, (h - c->cy) / c->fy);
  c->lim_yn = fmaf(0.3f, tan_y, c->cy / c->fy);
}

typedef struct vo_record {
  float mean_x, mean_y, conic0, conic1, conic2, opacity, depth;
  float rgb[3];
  int64_t gid;
  int radius_x, radius_y;
  int min_tx, min_ty, max_tx, max_ty;
  /* exact-ray mode: camera-space precision (upper triangle), precision * mean
   * and mean^T precision mean, all rounded from double */
  float prec[6], prec_mean[3], mean_prec_mean;
} vo_record;

static int project(const vo_scene* s, int64_t g, const cam_const* c, float near_plane,
                   float far_plane, float sigma, float eps, int antialiased, int ray_eval,
                   vo_record* out, float* pxyz) {
  float o = s->opacities[g];
  if (!(o >= ALPHA_THRESHOLD)) return 0;
  const float mx = s->means[g * 3 + 0], my = s->means[g * 3 + 1], mz = s->means[g * 3 + 2];
  const float pz = fmaf(c->r[8], mz, fmaf(c->r[7], my, fmaf(c->r[6], mx, c->t[2])));
  if (pz < near_plane || pz > far_plane) return 0;
  const float px = fmaf(c->r[2], mz, fmaf(c->r[1], my, fmaf(c->r[0], mx, c->t[0])));
  const float py = fmaf(c->r[5], mz, fmaf(c->r[4], my, fmaf(c->r[3], mx, c->t[1])));
  const float iz = 1.0f / pz;
  const float u = fmaf(c->fx * px, iz, c->cx);
  const float v = fmaf(c->fy * py, iz, c->cy);
  const float* cv = s->covariances + g * 6;
  const float s00 = cv[0], s01 = cv[1], s02 = cv[2], s11 = cv[3], s12 = cv[4], s22 = cv[5];
  float tm[9];
  for (int row = 0; row < 3; ++row) {
    const float r0 = c->r[row * 3 + 0], r1 = c->r[row * 3 + 1], r2 = c->r[row * 3 + 2];
    tm[row * 3 + 0] = fmaf(r2, s02, fmaf(r1, s01, r0 * s00));
    tm[row * 3 + 1] = fmaf(r2, s12, fmaf(r1, s11, r0 * s01));
    tm[row * 3 + 2] = fmaf(r2, s22, fmaf(r1, s12, r0 * s02));
  }
#define VO_COV(i, j)                                                    \
  fmaf(tm[i * 3 + 2], c->r[j * 3 + 2],                                  \
       fmaf(tm[i * 3 + 1], c->r[j * 3 + 1], tm[i * 3 + 0] * c->r[j * 3 + 0]))
  const float c00 = VO_COV(0, 0), c01 = VO_COV(0, 1), c02 = VO_COV(0, 2);
  const float c11 = VO_COV(1, 1), c12 = VO_COV(1, 2), c22 = VO_COV(2, 2);
#undef VO_COV
  const float tx = px * iz, ty = py * iz;
  const float clx = pz * fminf(c->lim_xp, fmaxf(-c->lim_xn, tx));
  const float cly = pz * fminf(c->lim_yp, fmaxf(-c->lim_yn, ty));
  const float iz2 = iz * iz;
  const float j00 = c->fx * iz;
  const float j02 = ((-c->fx) * clx) * iz2;
  const float j11 = c->fy * iz;
  const float j12 = ((-c->fy) * cly) * iz2;
  const float a_raw = fmaf(j02 * j02, c22, fmaf((2.0f * j00) * j02, c02, (j00 * j00) * c00));
  const float b = fmaf(j02 * j12, c22, fmaf(j02 * j11, c12, fmaf(j00 * j12, c02, (j00 * j11) * c01)));
  const float c_raw = fmaf(j12 * j12, c22, fmaf((2.0f * j11) * j12, c12, (j11 * j11) * c11));
  const float a = a_raw + eps;
  const float cc = c_raw + eps;
  const float det = fmaf(a, cc, -(b * b));
  if (!(det > 0.0f)) return 0;
  if (antialiased) {
    const float det_raw = fmaf(a_raw, c_raw, -(b * b));
    const float floor2 = MIN_AA_COMPENSATION * MIN_AA_COMPENSATION;
    const float comp = sqrtf(fmaxf(floor2, det_raw / det));
    o = o * comp;
    if (!(o >= ALPHA_THRESHOLD)) return 0;
  }
  const float ext_o = sqrtf(2.0f * vo_log(o / ALPHA_THRESHOLD));
  const float ext = fminf(sigma, ext_o);
  int rx = ceil_radius(ext * sqrtf(a));
  int ry = ceil_radius(ext * sqrtf(cc));
  if (rx <= 0 && ry <= 0) return 0;
  float cull_x = u, cull_y = v;
  if (ray_eval) {
    /* Exact ray evaluation: precision of the camera-space covariance and the
     * image-plane ellipse where a pixel ray's Mahalanobis distance to the
     * mean is at most sigma (renderer_cuda.cu:795-948), in double. */
    const double d00 = c00, d01 = c01, d02 = c02, d11 = c11, d12 = c12, d22 = c22;
    const double det3 = d00 * (d11 * d22 - d12 * d12) - d01 * (d01 * d22 - d02 * d12) +
                        d02 * (d01 * d12 - d02 * d11);
    if (!(det3 > 1.0e-48)) return 0;
    const double inv3 = 1.0 / det3;
    const double p00 = (d11 * d22 - d12 * d12) * inv3;
    const double p01 = (d02 * d12 - d01 * d22) * inv3;
    const double p02 = (d01 * d12 - d02 * d11) * inv3;
    const double p11 = (d00 * d22 - d02 * d02) * inv3;
    const double p12 = (d01 * d02 - d00 * d12) * inv3;
    const double p22 = (d00 * d11 - d01 * d01) * inv3;
    const double x = px, y = py, z = pz;
    const double m0 = p00 * x + p01 * y + p02 * z;
    const double m1 = p01 * x + p11 * y + p12 * z;
    const double m2 = p02 * x + p12 * y + p22 * z;
    const double mpm = x * m0 + y * m1 + z * m2;
    out->prec[0] = (float)p00;
    out->prec[1] = (float)p01;
    out->prec[2] = (float)p02;
    out->prec[3] = (float)p11;
    out->prec[4] = (float)p12;
    out->prec[5] = (float)p22;
    out->prec_mean[0] = (float)m0;
    out->prec_mean[1] = (float)m1;
    out->prec_mean[2] = (float)m2;
    out->mean_prec_mean = (float)mpm;
    const double q = mpm - (double)sigma * (double)sigma;
    const double k00 = q * p00 - m0 * m0, k01 = q * p01 - m0 * m1, k02 = q * p02 - m0 * m2;
    const double k11 = q * p11 - m1 * m1, k12 = q * p12 - m1 * m2, k22 = q * p22 - m2 * m2;
    const double kdet = k00 * k11 - k01 * k01;
    int finite = 0;
    if (k00 > 0.0 && kdet > 0.0) {
      const double ikd = 1.0 / kdet;
      const double cxn = (k01 * k12 - k11 * k02) * ikd;
      const double cyn = (k01 * k02 - k00 * k12) * ikd;
      const double scale = -(k22 + k02 * cxn + k12 * cyn);
      if (scale > 0.0) {
        const double exn = sqrt(scale * k11 * ikd);
        const double eyn = sqrt(scale * k00 * ikd);
        const double cmx = (double)c->fx * cxn + (double)c->cx;
        const double cmy = (double)c->fy * cyn + (double)c->cy;
        cull_x = (float)cmx;
        cull_y = (float)cmy;
        const int erx = saturating_int(ceilf((float)(fabs((double)c->fx) * exn)));
        const int ery = saturating_int(ceilf((float)(fabs((double)c->fy) * eyn)));
        rx = erx > 1 ? erx : 1;
        ry = ery > 1 ? ery : 1;
        finite = isfinite(cmx) && isfinite(cmy) && isfinite(exn) && isfinite(eyn);
      }
    }
    if (!finite) {
      const int full = (int)c->width > (int)c->height ? (int)c->width : (int)c->height;
      cull_x = 0.5f * c->width;
      cull_y = 0.5f * c->height;
      rx = full;
      ry = full;
    }
  }
  const float frx = (float)rx, fry = (float)ry;
  if (cull_x + frx <= 0.0f || cull_y + fry <= 0.0f || cull_x - frx >= c->width ||
      cull_y - fry >= c->height) {
    return 0;
  }
  const float idet = 1.0f / det;
  out->mean_x = cull_x;
  out->mean_y = cull_y;
  out->conic0 = cc * idet;
  out->conic1 = (-b) * idet;
  out->conic2 = a * idet;
  out->opacity = fminf(fmaxf(o, 0.0f), 1.0f);
  out->depth = pz;
  out->gid = g;
  out->radius_x = rx;
  out->radius_y = ry;
  pxyz[0] = px;
  pxyz[1] = py;
  pxyz[2] = pz;
  return 1;
}

static void eval_sh(int degree, const float* coeffs, const cam_const* c, const float* p,
                    float* rgb) {
  const float px = p[0], py = p[1], pz = p[2];
  const float dx = fmaf(c->r[6], pz, fmaf(c->r[3], py, c->r[0] * px));
  const float dy = fmaf(c->r[7], pz, fmaf(c->r[4], py, c->r[1] * px));
  const float dz = fmaf(c->r[8], pz, fmaf(c->r[5], py, c->r[2] * px));
  const float inv = 1.0f / sqrtf(fmaf(dz, dz, fmaf(dy, dy, dx * dx)));
  const float x = dx * inv, y = dy * inv, z = dz * inv;
  float basis[16];
  int count = 1;
  basis[0] = 0.28209479177387814f;
  if (degree >= 1) {
    basis[1] = -0.4886025119029199f * y;
    basis[2] = 0.4886025119029199f * z;
    basis[3] = -0.4886025119029199f * x;
    count = 4;
  }
  const float xx = x * x, yy = y * y, zz = z * z, xy = x * y, yz = y * z, xz = x * z;
  if (degree >= 2) {
    basis[4] = 1.0925484305920792f * xy;
    basis[5] = -1.0925484305920792f * yz;
    basis[6] = 0.31539156525252005f * ((2.0f * zz - xx) - yy);
    basis[7] = -1.0925484305920792f * xz;
    basis[8] = 0.5462742152960396f * (xx - yy);
    count = 9;
  }
  if (degree >= 3) {
    basis[9] = (-0.5900435899266435f * y) * (3.0f * xx - yy);
    basis[10] = (2.890611442640554f * xy) * z;
    basis[11] = (-0.4570457994644658f * y) * ((4.0f * zz - xx) - yy);
    basis[12] = (0.3731763325901154f * z) * ((2.0f * zz - 3.0f * xx) - 3.0f * yy);
    basis[13] = (-0.4570457994644658f * x) * ((4.0f * zz - xx) - yy);
    basis[14] = (1.445305721320277f * z) * (xx - yy);
    basis[15] = (-0.5900435899266435f * x) * (xx - 3.0f * yy);
    count = 16;
  }
  for (int ch = 0; ch < 3; ++ch) {
    float acc = basis[0] * coeffs[ch];
    for (int k = 1; k < count; ++k) acc = fmaf(basis[k], coeffs[k * 3 + ch], acc);
    rgb[ch] = fmaxf(acc + 0.5f, 0.0f);
  }
}

typedef struct vo_entry {
  uint32_t tile;      /* global tile */
  uint32_t depth_bits;
  uint32_t gid;
  uint32_t slot;      /* active slot (duplicate cameras) */
  uint32_t record;    /* index into the record array */
} vo_entry;

static int entry_cmp(const void* pa, const void* pb) {
  const vo_entry* a = (const vo_entry*)pa;
  const vo_entry* b = (const vo_entry*)pb;
  if (a->tile != b->tile) return a->tile < b->tile ? -1 : 1;
  if (a->depth_bits != b->depth_bits) return a->depth_bits < b->depth_bits ? -1 : 1;
  if (a->gid != b->gid) return a->gid < b->gid ? -1 : 1;
  if (a->slot != b->slot) return a->slot < b->slot ? -1 : 1;
  return 0;
}

/* Optional per-pixel decision margins of the screen-space compositor, three
 * floats per pixel (NULL: not written).  For each pixel: the smallest
 * relative distance of an evaluated record's unclamped alpha o exp(power)
 * from the 1/255 floor, and of its power from the -20 cut; the smallest
 * relative distance of a running transmittance T (1 - alpha) from the 1e-4
 * stop; and the smallest relative depth gap between two consecutive blended
 * records.  A pixel whose margins are all large cannot change when an
 * implementation evaluates the same equation with a few ulp of different
 * rounding (fast-math exp or division, contracted products); a small margin
 * marks a decision that can go the other way, or two records whose order
 * can swap.  Test instrumentation only; set with vo_set_margin_output and
 * reset to NULL after the render. */
static float* g_margins = NULL;
void vo_set_margin_output(float* margins) { g_margins = margins; }

static float rel_gap(float a, float b) {
  const float d = fabsf(a - b);
  const float m = fmaxf(fabsf(a), fabsf(b));
  return m > 0.0f ? d / m : 0.0f;
}

typedef struct slot_info {
  int valid, slot_scene, width, height, tiles_x, tiles_y;
  int64_t camera, g_begin, g_count, tile_base, pixel_base;
} slot_info;

/* Renders every active camera; returns 0, or -1 on allocation failure.
 * tile_counts (global tiles) and sorted_gaussian_ids (in global sorted order,
 * up to sorted_capacity entries) are optional outputs for parity checks. */
int vo_render(const vo_scene* s, const vo_cameras* cams, const vo_options* opt, float* rgb,
              float* depth, float* alpha, int64_t* semantic, int32_t* tile_counts,
              int64_t tile_count_capacity, int32_t* sorted_gaussian_ids,
              int64_t sorted_capacity, vo_stats* stats) {
#ifdef _OPENMP
  if (opt->threads > 0) omp_set_num_threads(opt->threads);
#endif
  /* Exact-ray mode bins 16-pixel tiles as 32-pixel tiles in the plain form
   * (renderer_cuda.cu:2670-2676). */
  const int ts = (opt->ray_eval && opt->tile_size == 16 && !cams->widths) ? 32 : opt->tile_size;
  const float near_f = (float)opt->near_plane, far_f = (float)opt->far_plane;
  const float sigma = (float)opt->support_sigma, eps = (float)opt->covariance_epsilon;
  const float its = 1.0f / (float)ts;
  const int64_t active = cams->active_ids ? cams->active_count : cams->batch;
  slot_info* slots = (slot_info*)calloc((size_t)(active > 0 ? active : 1), sizeof(slot_info));
  if (!slots) return -1;
  for (int64_t a = 0; a < active; ++a) {
    slot_info* si = &slots[a];
    const int64_t cam = cams->active_ids ? cams->active_ids[a] : a;
    si->valid = cam >= 0 && cam < cams->batch;
    si->slot_scene = -1;
    if (!si->valid) continue;
    si->camera = cam;
    for (int64_t k = 0; k < s->scene_count; ++k) {
      if (s->registered_scene_ids[k] == cams->camera_scene_ids[cam]) {
        si->slot_scene = (int)k;
        break;
      }
    }
    if (si->slot_scene >= 0) {
      si->g_begin = s->scene_offsets[si->slot_scene];
      si->g_count = s->scene_offsets[si->slot_scene + 1] - si->g_begin;
    }
    if (cams->widths) {
      si->width = cams->widths[cam];
      si->height = cams->heights[cam];
    } else {
      si->width = (int)opt->width;
      si->height = (int)opt->height;
    }
    si->tiles_x = (si->width + ts - 1) / ts;
    si->tiles_y = (si->height + ts - 1) / ts;
    if (cams->widths) {
      si->tile_base = cams->tile_offsets[cam];
      si->pixel_base = cams->pixel_offsets[cam];
    } else {
      si->tile_base = cam * (int64_t)si->tiles_x * si->tiles_y;
      si->pixel_base = cam * (int64_t)si->width * si->height;
    }
  }

  /* Projection, per slot in order, Gaussians ascending. */
  int64_t total_records = 0;
  int64_t record_cap = 1024;
  vo_record* records = (vo_record*)malloc((size_t)record_cap * sizeof(vo_record));
  int64_t entry_count = 0, entry_cap = 4096;
  vo_entry* entries = (vo_entry*)malloc((size_t)entry_cap * sizeof(vo_entry));
  if (!records || !entries) return -1;
  for (int64_t a = 0; a < active; ++a) {
    const slot_info* si = &slots[a];
    if (!si->valid || si->slot_scene < 0 || si->g_count <= 0) continue;
    cam_const c;
    make_cam_const(cams->viewmats + si->camera * 16, cams->env_xforms + si->camera * 16,
                   cams->intrinsics + si->camera * 9, si->width, si->height, &c);
    vo_record* local = (vo_record*)malloc((size_t)si->g_count * sizeof(vo_record));
    char* vis = (char*)calloc((size_t)si->g_count, 1);
    if (!local || !vis) return -1;
#pragma omp parallel for schedule(dynamic, 4096)
    for (int64_t i = 0; i < si->g_count; ++i) {
      const int64_t g = si->g_begin + i;
      float p[3];
      vo_record r;
      if (!project(s, g, &c, near_f, far_f, sigma, eps, opt->antialiased, opt->ray_eval, &r, p)) continue;
      if (opt->sh_degree < 0) {
        r.rgb[0] = s->features[g * s->feature_width + 0];
        r.rgb[1] = s->features[g * s->feature_width + 1];
        r.rgb[2] = s->features[g * s->feature_width + 2];
      } else {
        eval_sh(opt->sh_degree, s->features + g * s->feature_width, &c, p, r.rgb);
      }
      const float frx = (float)r.radius_x, fry = (float)r.radius_y;
      r.min_tx = floor_clamped(r.mean_x * its - frx * its);
      r.min_ty = floor_clamped(r.mean_y * its - fry * its);
      r.max_tx = ceil_clamped(r.mean_x * its + frx * its);
      r.max_ty = ceil_clamped(r.mean_y * its + fry * its);
      if (r.min_tx < 0) r.min_tx = 0;
      if (r.min_ty < 0) r.min_ty = 0;
      if (r.max_tx > si->tiles_x) r.max_tx = si->tiles_x;
      if (r.max_ty > si->tiles_y) r.max_ty = si->tiles_y;
      local[i] = r;
      vis[i] = 1;
    }
    for (int64_t i = 0; i < si->g_count; ++i) {
      if (!vis[i]) continue;
      if (total_records == record_cap) {
        record_cap *= 2;
        records = (vo_record*)realloc(records, (size_t)record_cap * sizeof(vo_record));
        if (!records) return -1;
      }
      const int64_t ri = total_records++;
      records[ri] = local[i];
      const vo_record* r = &records[ri];
      for (int ty = r->min_ty; ty < r->max_ty; ++ty) {
        for (int tx = r->min_tx; tx < r->max_tx; ++tx) {
          if (entry_count == entry_cap) {
            entry_cap *= 2;
            entries = (vo_entry*)realloc(entries, (size_t)entry_cap * sizeof(vo_entry));
            if (!entries) return -1;
          }
          vo_entry* e = &entries[entry_count++];
          e->tile = (uint32_t)(si->tile_base + (int64_t)ty * si->tiles_x + tx);
          e->depth_bits = float_to_bits(r->depth);
          e->gid = (uint32_t)r->gid;
          e->slot = (uint32_t)a;
          e->record = (uint32_t)ri;
        }
      }
    }
    free(local);
    free(vis);
  }
  qsort(entries, (size_t)entry_count, sizeof(vo_entry), entry_cmp);

  /* Tile ranges over the sorted entries. */
  int64_t active_tiles = 0;
  for (int64_t i = 0; i < entry_count; ++i) {
    if (i == 0 || entries[i - 1].tile != entries[i].tile) ++active_tiles;
    if (tile_counts && (int64_t)entries[i].tile < tile_count_capacity) tile_counts[entries[i].tile] += 1;
    if (sorted_gaussian_ids && i < sorted_capacity) sorted_gaussian_ids[i] = (int32_t)entries[i].gid;
  }
  if (stats) {
    stats->visible = total_records;
    stats->intersections = entry_count;
    stats->active_tiles = active_tiles;
  }

  /* Compositor, per slot and tile. */
  const float sem_min = (float)opt->semantic_min_alpha;
  for (int64_t a = 0; a < active; ++a) {
    const slot_info* si = &slots[a];
    if (!si->valid) continue;
    const int64_t tiles = (int64_t)si->tiles_x * si->tiles_y;
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t t = 0; t < tiles; ++t) {
      const uint32_t gt = (uint32_t)(si->tile_base + t);
      /* Binary search of the tile's range in the sorted entries. */
      int64_t lo = 0, hi = entry_count;
      while (lo < hi) {
        const int64_t mid = (lo + hi) / 2;
        if (entries[mid].tile < gt) lo = mid + 1; else hi = mid;
      }
      const int64_t start = lo;
      hi = entry_count;
      while (lo < hi) {
        const int64_t mid = (lo + hi) / 2;
        if (entries[mid].tile <= gt) lo = mid + 1; else hi = mid;
      }
      const int64_t end = lo;
      const int tx0 = (int)(t % si->tiles_x) * ts;
      const int ty0 = (int)(t / si->tiles_x) * ts;
      for (int ly = 0; ly < ts; ++ly) {
        for (int lx = 0; lx < ts; ++lx) {
          const int x = tx0 + lx, y = ty0 + ly;
          if (x >= si->width || y >= si->height) continue;
          const float cx = (float)x + 0.5f, cy = (float)y + 0.5f;
          float tr = 1.0f, r = 0.0f, g = 0.0f, b = 0.0f, dep = 0.0f, best_w = -1.0f;
          int64_t best_sem = -1;
          if (opt->ray_eval) {
            /* Exact ray evaluation (renderer_cuda.cu:203-245,2190-2270): the
             * pixel ray's Mahalanobis distance to each mean, no 1/255 cut or
             * 0.99 clamp, and the record that takes T to 1e-4 is blended. */
            const float* in = cams->intrinsics + si->camera * 9;
            const float ray_x = (cx - in[2]) / in[0];
            const float ray_y = (cy - in[5]) / in[4];
            const float s2 = sigma * sigma;
            for (int64_t i = start; i < end; ++i) {
              const vo_record* rec = &records[entries[i].record];
              /* Only pixels inside the box of the record's ray ellipse
               * (radius + 1 px around its centre; 16-bit, 32767 unbounded). */
              const int bx = (rec->radius_x < 32766 ? rec->radius_x : 32766) + 1;
              const int by = (rec->radius_y < 32766 ? rec->radius_y : 32766) + 1;
              const float hx = bx >= 32767 ? INFINITY : (float)bx;
              const float hy = by >= 32767 ? INFINITY : (float)by;
              if (fabsf(cx - rec->mean_x) > hx || fabsf(cy - rec->mean_y) > hy) continue;
              const float* P = rec->prec;
              const float rpr = fmaf(2.0f * P[4], ray_y,
                                     fmaf(P[3] * ray_y, ray_y,
                                          fmaf(2.0f * P[2], ray_x,
                                               fmaf((2.0f * P[1]) * ray_x, ray_y, (P[0] * ray_x) * ray_x)))) +
                                P[5];
              if (!(rpr > 0.0f)) continue;
              const float rpm = fmaf(ray_y, rec->prec_mean[1], ray_x * rec->prec_mean[0]) + rec->prec_mean[2];
              const float m2 = fmaxf(0.0f, rec->mean_prec_mean - (rpm * rpm) / rpr);
              if (m2 > s2 || m2 > 174.0f) continue; /* exp below float range: no contribution */
              const float al = fminf(1.0f, rec->opacity * vo_exp(-0.5f * m2));
              if (!(al > 0.0f)) continue;
              const float next_t = tr * (1.0f - al);
              const float w = tr * al;
              r = fmaf(w, rec->rgb[0], r);
              g = fmaf(w, rec->rgb[1], g);
              b = fmaf(w, rec->rgb[2], b);
              dep = fmaf(w, rec->depth, dep);
              if (w > best_w) {
                best_w = w;
                best_sem = s->semantic_ids[rec->gid];
              }
              tr = next_t;
              if (next_t <= TRANSMITTANCE_THRESHOLD) break;
            }
          }
          float m_alpha = INFINITY, m_trans = INFINITY, m_depth = INFINITY, last_depth = NAN;
          for (int64_t i = start; i < end && !opt->ray_eval; ++i) {
            const vo_record* rec = &records[entries[i].record];
            const float dx = cx - rec->mean_x;
            const float dy = cy - rec->mean_y;
            const float q = fmaf(rec->conic2 * dy, dy,
                                 fmaf((2.0f * rec->conic1) * dx, dy, (rec->conic0 * dx) * dx));
            const float power = -0.5f * q;
            if (g_margins && power <= 0.0f) m_alpha = fminf(m_alpha, rel_gap(power, -20.0f));
            if (power > 0.0f || power < -20.0f) continue;
            const float raw = rec->opacity * vo_exp(power);
            if (g_margins) m_alpha = fminf(m_alpha, rel_gap(raw, ALPHA_THRESHOLD));
            const float al = fminf(MAX_ALPHA, raw);
            if (al < ALPHA_THRESHOLD) continue;
            const float next_t = tr * (1.0f - al);
            if (g_margins) {
              m_trans = fminf(m_trans, rel_gap(next_t, TRANSMITTANCE_THRESHOLD));
              if (last_depth == last_depth) m_depth = fminf(m_depth, rel_gap(rec->depth, last_depth));
              last_depth = rec->depth;
            }
            if (next_t <= TRANSMITTANCE_THRESHOLD) break;
            const float w = tr * al;
            r = fmaf(w, rec->rgb[0], r);
            g = fmaf(w, rec->rgb[1], g);
            b = fmaf(w, rec->rgb[2], b);
            dep = fmaf(w, rec->depth, dep);
            if (w > best_w) {
              best_w = w;
              best_sem = s->semantic_ids[rec->gid];
            }
            tr = next_t;
          }
          const int64_t pix = si->pixel_base + (int64_t)y * si->width + x;
          if (g_margins) {
            g_margins[pix * 3 + 0] = m_alpha;
            g_margins[pix * 3 + 1] = m_trans;
            g_margins[pix * 3 + 2] = m_depth;
          }
          const float out_alpha = 1.0f - tr;
          if (opt->output_srgb) {
            r = vo_srgb(r);
            g = vo_srgb(g);
            b = vo_srgb(b);
          }
          rgb[pix * 3 + 0] = r;
          rgb[pix * 3 + 1] = g;
          rgb[pix * 3 + 2] = b;
          if (opt->full_sensor_output) {
            alpha[pix] = out_alpha;
            depth[pix] = out_alpha > 1.0e-8f ? dep / out_alpha : INFINITY;
            semantic[pix] = (best_w >= 0.0f && out_alpha >= sem_min) ? best_sem : -1;
          }
        }
      }
    }
  }
  free(records);
  free(entries);
  free(slots);
  return 0;
}

/* Exposed for unit tests of the polynomial methods. */
float vo_exp_public(float x) { return vo_exp(x); }
float vo_log_public(float y) { return vo_log(y); }
float vo_srgb_public(float v) { return vo_srgb(v); }
