// Shared device helpers of the B200 renderer.
//
// Arithmetic contract: every floating-point operation whose result reaches a
// tile ID, a key, a blend weight or an output pixel is written as an explicit
// IEEE round-to-nearest intrinsic (__fmul_rn, __fadd_rn, __fsub_rn,
// __fmaf_rn, __fdiv_rn, __fsqrt_rn).  The compiler can therefore neither
// contract nor approximate it, and a C restatement that performs the same
// operations in the same order (fmaf, *, +, /, sqrtf with contraction off)
// reproduces every bit.  exp and log are evaluated by the polynomial methods
// below (not CUDA's math library) for the same reason.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace vgr {

constexpr float kAlphaThreshold = 1.0f / 255.0f;   // renderer_cuda.cu:24
constexpr float kMaxAlpha = 0.99f;                 // renderer_cuda.cu:25
constexpr float kTransmittanceThreshold = 1.0e-4f; // renderer_cuda.cu:23
constexpr float kMinAntialiasCompensation = 0.005f;// renderer_cuda.cu:26

__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float ffma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ float fdiv(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ float fsqrt(float a) { return __fsqrt_rn(a); }
// Double-precision counterparts (the exact-ray projection works in double).
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double ddiv(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ double dsqrt(double a) { return __dsqrt_rn(a); }

// exp(x) for finite x in [-87, 88]: Cody-Waite reduction x = n ln2 + r with
// n = rint(x log2 e), r carried as f = x log2(e) - n in two fma steps, and a
// degree-5 minimax polynomial of 2^f on |f| <= 0.5 (Remez exchange for the
// relative error, 7.5e-8; coefficients from exp2_minimax.py, rounded to
// float), scaled by 2^n through the exponent field: within 2.3e-7 of exp
// over the range.  The rounding to an integer adds and subtracts 1.5 * 2^23
// (round-to-nearest-even, exact for |t| < 2^22, so identical to rint), and
// n's integer value is read from the bits of the sum: all on the FMA and
// integer pipes.
__device__ __forceinline__ float vexp(float x) {
  const float kLog2eHi = 1.44269502162933349609375f;
  const float kLog2eLo = 1.925963033500011079e-8f;
  const float kRoundMagic = 12582912.0f;  // 1.5 * 2^23
  const float t = fmul(x, kLog2eHi);
  const float tm = fadd(t, kRoundMagic);
  const float n = fsub(tm, kRoundMagic);
  float f = ffma(x, kLog2eHi, -n);
  f = ffma(x, kLog2eLo, f);
  float p = 1.327647245e-03f;        // c5
  p = ffma(p, f, 9.675540961e-03f);  // c4
  p = ffma(p, f, 5.550713092e-02f);  // c3
  p = ffma(p, f, 2.402212024e-01f);  // c2
  p = ffma(p, f, 6.931469440e-01f);  // c1
  p = ffma(p, f, 1.000000119e+00f);  // c0
  const int e = __float_as_int(tm) - 0x4b400000;  // bits of 1.5 * 2^23
  return fmul(p, __int_as_float((e + 127) << 23));
}

// One 256-bit read-only load of eight floats (p 32-byte aligned).
__device__ __forceinline__ void ldg8(const float* p, float (&v)[8]) {
  asm("ld.global.nc.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
      : "=f"(v[0]), "=f"(v[1]), "=f"(v[2]), "=f"(v[3]), "=f"(v[4]), "=f"(v[5]), "=f"(v[6]), "=f"(v[7])
      : "l"(p));
}

// ln(y) for positive normal finite y: y = m 2^e with m in [sqrt(1/2), sqrt(2)),
// ln m = 2 atanh(s), s = (m-1)/(m+1), atanh by its odd series through s^11
// (|s| <= 0.1716, truncation < 1e-10 relative), ln 2 split in two parts.
__device__ __forceinline__ float vlog(float y) {
  const int bits = __float_as_int(y);
  int e = ((bits >> 23) & 0xff) - 127;
  float m = __int_as_float((bits & 0x007fffff) | 0x3f800000);
  if (m > 1.41421353816986083984375f) {
    m = fmul(m, 0.5f);
    e += 1;
  }
  const float s = fdiv(fsub(m, 1.0f), fadd(m, 1.0f));
  const float s2 = fmul(s, s);
  float p = 0.0909090909090909f;               // 1/11
  p = ffma(p, s2, 0.1111111111111111f);        // 1/9
  p = ffma(p, s2, 0.1428571428571428f);        // 1/7
  p = ffma(p, s2, 0.2f);                       // 1/5
  p = ffma(p, s2, 0.3333333333333333f);        // 1/3
  p = ffma(p, s2, 1.0f);
  const float lnm = fmul(fmul(2.0f, s), p);
  const float fe = static_cast<float>(e);
  const float kLn2Hi = 0.693145751953125f;
  const float kLn2Lo = 1.428606765330187e-06f;
  return ffma(fe, kLn2Hi, ffma(fe, kLn2Lo, lnm));
}

// sRGB transfer (renderer_cuda.cu:161-166) with pow(v, 1/2.4) as
// vexp(vlog(v) / 2.4).
__device__ __forceinline__ float linear_to_srgb(float v) {
  v = fminf(fmaxf(v, 0.0f), 1.0f);
  if (v <= 0.0031308f) {
    return fmul(12.92f, v);
  }
  const float p = vexp(fmul(vlog(v), 0.4166666666666667f));
  return fsub(fmul(1.055f, p), 0.055f);
}

// Float -> int conversions with explicit saturation, so the C restatement
// (which has no saturating conversion) agrees for out-of-range values.
__device__ __forceinline__ int ceil_radius(float x) {
  return x > 0.0f ? static_cast<int>(fminf(ceilf(x), 2147483520.0f)) : 0;
}
__device__ __forceinline__ int floor_clamped(float x) {
  // NaN compares false and maps to 0.
  if (!(x == x)) return 0;
  return static_cast<int>(floorf(fminf(fmaxf(x, -1073741824.0f), 1073741824.0f)));
}
__device__ __forceinline__ int ceil_clamped(float x) {
  if (!(x == x)) return 0;
  return static_cast<int>(ceilf(fminf(fmaxf(x, -1073741824.0f), 1073741824.0f)));
}

__device__ __forceinline__ uint64_t ld_acquire_u64(const uint64_t* p) {
  uint64_t v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_u64(uint64_t* p, uint64_t v) {
  asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ uint32_t lanemask_lt() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// Bounded spin budget for decoupled look-back waits.  A wait that runs out
// records VGR_DEVICE_ERROR_LOOKBACK in the device status word and the kernel
// continues with a clamped result (outputs are then invalid but no access
// leaves its buffer).
constexpr uint32_t kSpinLimit = 1u << 22;
constexpr int kDeviceErrorLookback = 1;

// Order-preserving map of a float to uint32 (unsigned comparison of the
// codes orders the floats) and its inverse.
__device__ __forceinline__ uint32_t float_order(float f) {
  const uint32_t u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float order_float(uint32_t u) {
  return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

// Spreads the low 10 bits of v to every third bit (one axis of a 30-bit
// Morton code).
__device__ __forceinline__ uint32_t expand_bits(uint32_t v) {
  v &= 0x000003ffu;
  v = (v | (v << 16)) & 0x030000ffu;
  v = (v | (v << 8)) & 0x0300f00fu;
  v = (v | (v << 4)) & 0x030c30c3u;
  v = (v | (v << 2)) & 0x09249249u;
  return v;
}

}  // namespace vgr
