// Scene and camera ingestion on the device: INRIA 3DGS PLY vertex rows ->
// renderer-ready canonical scene tensors, and USD (row-vector) camera world
// matrices -> OpenCV view matrices.
//
// PLY canonicalisation follows src/isaacsim_gaussian_renderer/ply_loader.py:
// load_ply_to_gaussians (:52-90: property selection, f_rest channel-major ->
// coefficient-major reorder, semantic_id or 0) and canonicalize_3dgs_scene
// (:93-135: scale = exp, opacity = sigmoid, quaternion / max(|q|, eps) with
// |q| <= eps -> identity, features[0..2] = clamp(0.5 + SH_C0 dc, 0, 1)).
// The reference parses with plyfile on the host and activates with torch
// operations; here one thread per vertex reads its packed row (any of the
// PLY scalar types, at the byte offsets of the header) and writes every
// output, so a scene is ingested in one pass over the file's bytes.
//
// Camera ingestion follows src/isaacsim_gaussian_renderer/
// fabric_camera_kernels.py:8-49 (world matrix rows -> R = rows with the y and
// z axes negated, t = -R * position), one thread per camera.
#include <cuda_runtime.h>

#include <climits>
#include <cstring>

#include "../../include/vgr_b200.h"
#include "vgr_api_internal.h"
#include "vgr_common.cuh"

namespace vgr {
namespace {

__device__ __forceinline__ double read_scalar(const unsigned char* p, int type) {
  // Rows are packed (no alignment): assemble the value from bytes.
  unsigned char b[8];
  const int size = (type == VGR_PLY_FLOAT64 || type == VGR_PLY_INT64) ? 8
                   : (type == VGR_PLY_INT16 || type == VGR_PLY_UINT16) ? 2
                   : (type == VGR_PLY_INT8 || type == VGR_PLY_UINT8)   ? 1
                                                                       : 4;
  for (int i = 0; i < size; ++i) b[i] = p[i];
  switch (type) {
    case VGR_PLY_FLOAT32: { float v; memcpy(&v, b, 4); return v; }
    case VGR_PLY_FLOAT64: { double v; memcpy(&v, b, 8); return v; }
    case VGR_PLY_INT8: { int8_t v; memcpy(&v, b, 1); return v; }
    case VGR_PLY_UINT8: { uint8_t v; memcpy(&v, b, 1); return v; }
    case VGR_PLY_INT16: { int16_t v; memcpy(&v, b, 2); return v; }
    case VGR_PLY_UINT16: { uint16_t v; memcpy(&v, b, 2); return v; }
    case VGR_PLY_INT32: { int32_t v; memcpy(&v, b, 4); return v; }
    case VGR_PLY_UINT32: { uint32_t v; memcpy(&v, b, 4); return v; }
    default: { int64_t v; memcpy(&v, b, 8); return static_cast<double>(v); }
  }
}

__device__ __forceinline__ int64_t read_integer(const unsigned char* p, int type) {
  if (type == VGR_PLY_INT64) {
    int64_t v;
    memcpy(&v, p, 8);  // byte copy: rows are unaligned
    return v;
  }
  return static_cast<int64_t>(read_scalar(p, type));
}

struct PlyParams {
  const unsigned char* rows;
  int64_t count;
  vgr_ply_layout layout;
  float* means;
  float* scales;
  float* rotations;
  float* opacities;
  float* features;
  int64_t feature_width;
  int64_t* semantic_ids;
};

constexpr int kPlyRows = 64;         // vertex rows per CTA
constexpr int kPlyMaxRowBytes = 512; // VGR_PLY_MAX_PROPERTIES x 8 bytes
constexpr int kPlyMaxStagedWidth = 64;

// One CTA per kPlyRows vertices: the CTA's rows (contiguous in the body) are
// staged into shared memory with 16-byte coalesced loads, each thread
// decodes its row from shared memory, and the feature rows (the bulk of the
// output) go back through shared memory so that their stores are coalesced
// too.  Dynamic shared memory sized to the file's row and feature widths
// (ply_smem_bytes): for the usual 62-float rows about 28 KB, eight CTAs per
// SM.
__host__ __device__ constexpr int64_t ply_rows_bytes(int64_t row_bytes) {
  return (kPlyRows * row_bytes + 15) / 16 * 16;
}
__host__ __device__ constexpr int64_t ply_smem_bytes(int64_t row_bytes, int64_t feature_width) {
  return ply_rows_bytes(row_bytes) +
         kPlyRows * (feature_width < kPlyMaxStagedWidth ? feature_width : kPlyMaxStagedWidth) * 4;
}

__global__ void __launch_bounds__(kPlyRows) ply_canonicalize_kernel(PlyParams p) {
  extern __shared__ __align__(16) unsigned char s_dyn[];
  const vgr_ply_layout& l = p.layout;
  unsigned char* s_rows = s_dyn;
  float* s_feat = reinterpret_cast<float*>(s_dyn + ply_rows_bytes(l.row_bytes));
  const int64_t g0 = static_cast<int64_t>(blockIdx.x) * kPlyRows;
  const int rows = static_cast<int>(min(static_cast<int64_t>(kPlyRows), p.count - g0));
  const int64_t bytes = static_cast<int64_t>(rows) * l.row_bytes;
  const unsigned char* src = p.rows + g0 * l.row_bytes;  // 16-byte aligned: 64 * row_bytes % 16 == 0
  const int64_t vec = bytes / 16;
  for (int64_t i = threadIdx.x; i < vec; i += kPlyRows) {
    reinterpret_cast<uint4*>(s_rows)[i] = __ldg(reinterpret_cast<const uint4*>(src) + i);
  }
  for (int64_t i = vec * 16 + threadIdx.x; i < bytes; i += kPlyRows) s_rows[i] = src[i];
  __syncthreads();

  const int t = threadIdx.x;
  const int64_t g = g0 + t;
  const bool live = t < rows;
  const unsigned char* row = s_rows + static_cast<int64_t>(t) * l.row_bytes;
  auto f = [&](int role) {
    const unsigned char* q = row + l.offsets[role];
    // float32 at a 4-byte-aligned offset (every property of the usual
    // all-float rows): one shared-memory word instead of four bytes.
    if (l.types[role] == VGR_PLY_FLOAT32 && (reinterpret_cast<uintptr_t>(q) & 3) == 0) {
      return *reinterpret_cast<const float*>(q);
    }
    return static_cast<float>(read_scalar(q, l.types[role]));
  };
  const int rest = l.rest_count;
  const int per_channel = rest / 3;
  const int width = static_cast<int>(p.feature_width);
  float dc[3] = {0.0f, 0.0f, 0.0f};
  int64_t semantic = 0;
  if (live) {
    for (int a = 0; a < 3; ++a) p.means[g * 3 + a] = f(VGR_PLY_X + a);
    for (int a = 0; a < 3; ++a) p.scales[g * 3 + a] = expf(f(VGR_PLY_SCALE0 + a));
    p.opacities[g] = 1.0f / (1.0f + expf(-f(VGR_PLY_OPACITY)));
    float q[4];
    for (int a = 0; a < 4; ++a) q[a] = f(VGR_PLY_ROT0 + a);
    const float norm = sqrtf(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
    const float eps = 1.1920928955078125e-07f;  // float32 machine epsilon
    for (int a = 0; a < 4; ++a) p.rotations[g * 4 + a] = norm <= eps ? (a == 0 ? 1.0f : 0.0f) : q[a] / norm;
    const float sh_c0 = 0.28209479177387814f;
    for (int c = 0; c < 3; ++c) dc[c] = fminf(fmaxf(0.5f + sh_c0 * f(VGR_PLY_DC0 + c), 0.0f), 1.0f);
    if (l.has_semantic) semantic = read_integer(row + l.offsets[VGR_PLY_SEMANTIC], l.types[VGR_PLY_SEMANTIC]);
    p.semantic_ids[g] = semantic;
  }
  // Feature rows: f_rest channel-major ([3, K-1]) -> coefficient-major,
  // assembled in shared memory and stored with coalesced writes (rows wider
  // than kPlyMaxStagedWidth are written directly).
  if (width > kPlyMaxStagedWidth) {
    if (live) {
      float* feat = p.features + g * p.feature_width;
      for (int c = 0; c < 3; ++c) feat[c] = dc[c];
      for (int k = 0; k < per_channel; ++k) {
        for (int c = 0; c < 3; ++c) feat[3 + k * 3 + c] = f(VGR_PLY_REST0 + c * per_channel + k);
      }
      for (int64_t i = 3 + rest; i < p.feature_width; ++i) feat[i] = 0.0f;
    }
    return;
  }
  if (live) {
    float* feat = s_feat + t * width;
    for (int c = 0; c < 3; ++c) feat[c] = dc[c];
    for (int k = 0; k < per_channel; ++k) {
      for (int c = 0; c < 3; ++c) feat[3 + k * 3 + c] = f(VGR_PLY_REST0 + c * per_channel + k);
    }
    for (int i = 3 + rest; i < width; ++i) feat[i] = 0.0f;
  }
  __syncthreads();
  float* dst = p.features + g0 * p.feature_width;
  const int n = rows * width;
  for (int i = threadIdx.x; i < n; i += kPlyRows) dst[i] = s_feat[i];
}

__global__ void __launch_bounds__(256) world_to_opencv_kernel(const double* __restrict__ world,
                                                              const int32_t* __restrict__ indices,
                                                              int64_t count, int64_t out_count,
                                                              float* __restrict__ viewmats,
                                                              int* __restrict__ bad) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const int32_t out = indices ? indices[i] : static_cast<int32_t>(i);
  if (out < 0 || out >= out_count) {
    atomicAdd(bad, 1);
    return;
  }
  const double* w = world + i * 16;  // row-vector convention: rows 0..2 axes, row 3 position
  const float px = static_cast<float>(w[12]), py = static_cast<float>(w[13]), pz = static_cast<float>(w[14]);
  float r[9];
  for (int c = 0; c < 3; ++c) {
    r[0 + c] = static_cast<float>(w[0 * 4 + c]);
    r[3 + c] = -static_cast<float>(w[1 * 4 + c]);
    r[6 + c] = -static_cast<float>(w[2 * 4 + c]);
  }
  float* v = viewmats + static_cast<int64_t>(out) * 16;
  for (int row = 0; row < 3; ++row) {
    v[row * 4 + 0] = r[row * 3 + 0];
    v[row * 4 + 1] = r[row * 3 + 1];
    v[row * 4 + 2] = r[row * 3 + 2];
    v[row * 4 + 3] = -(r[row * 3 + 0] * px + r[row * 3 + 1] * py + r[row * 3 + 2] * pz);
  }
  v[12] = 0.0f;
  v[13] = 0.0f;
  v[14] = 0.0f;
  v[15] = 1.0f;
}

}  // namespace
}  // namespace vgr

using vgr::fail;

extern "C" int vgr_ply_canonicalize(const void* vertex_rows, int64_t count,
                                    const vgr_ply_layout* layout, float* means, float* scales,
                                    float* rotations, float* opacities, float* features,
                                    int64_t feature_width, int64_t* semantic_ids, void* stream) {
  if (!vertex_rows || !layout || !means || !scales || !rotations || !opacities || !features ||
      !semantic_ids) {
    return fail(VGR_ERR_INVALID_ARGUMENT, "PLY ingestion arguments must be non-null");
  }
  if (count <= 0 || count > INT_MAX) return fail(VGR_ERR_INVALID_ARGUMENT, "vertex count must be in [1, INT_MAX]");
  if (layout->row_bytes <= 0) return fail(VGR_ERR_INVALID_ARGUMENT, "row_bytes must be positive");
  if (layout->rest_count < 0 || layout->rest_count % 3 != 0 ||
      layout->rest_count > VGR_PLY_MAX_PROPERTIES - VGR_PLY_REST0) {
    return fail(VGR_ERR_INVALID_ARGUMENT,
                "Expected an RGB-multiple number of f_rest fields, got %d.", layout->rest_count);
  }
  if (feature_width < 3 + layout->rest_count) {
    return fail(VGR_ERR_INVALID_ARGUMENT, "features are narrower than 3 + f_rest fields");
  }
  const int roles = VGR_PLY_REST0 + layout->rest_count;
  for (int r = 0; r < roles; ++r) {
    if (r == VGR_PLY_SEMANTIC && !layout->has_semantic) continue;
    const int t = layout->types[r];
    const int size = (t == VGR_PLY_FLOAT64 || t == VGR_PLY_INT64) ? 8
                     : (t == VGR_PLY_INT16 || t == VGR_PLY_UINT16) ? 2
                     : (t == VGR_PLY_INT8 || t == VGR_PLY_UINT8)   ? 1
                                                                   : 4;
    if (t < VGR_PLY_INT8 || t > VGR_PLY_FLOAT64 || layout->offsets[r] < 0 ||
        layout->offsets[r] + size > layout->row_bytes) {
      return fail(VGR_ERR_INVALID_ARGUMENT, "PLY property %d lies outside its vertex row", r);
    }
  }
  vgr::PlyParams p{};
  p.rows = static_cast<const unsigned char*>(vertex_rows);
  p.count = count;
  p.layout = *layout;
  p.means = means;
  p.scales = scales;
  p.rotations = rotations;
  p.opacities = opacities;
  p.features = features;
  p.feature_width = feature_width;
  p.semantic_ids = semantic_ids;
  if (layout->row_bytes > vgr::kPlyMaxRowBytes) {
    return fail(VGR_ERR_INVALID_ARGUMENT, "PLY vertex rows above %d bytes are not supported",
                vgr::kPlyMaxRowBytes);
  }
  if ((reinterpret_cast<uintptr_t>(vertex_rows) & 15) != 0) {
    return fail(VGR_ERR_INVALID_ARGUMENT, "vertex rows must start on a 16-byte boundary");
  }
  vgr::ply_canonicalize_kernel<<<static_cast<unsigned>((count + vgr::kPlyRows - 1) / vgr::kPlyRows),
                                 vgr::kPlyRows,
                                 static_cast<size_t>(vgr::ply_smem_bytes(layout->row_bytes, feature_width)),
                                 static_cast<cudaStream_t>(stream)>>>(p);
  return vgr::check_launch("PLY canonicalize");
}

extern "C" int vgr_world_to_opencv_viewmats(const double* world_matrices,
                                            const int32_t* camera_indices, int64_t count,
                                            float* viewmats, int64_t viewmat_count,
                                            int32_t* invalid_index_count, void* stream) {
  if (!world_matrices || !viewmats || !invalid_index_count) {
    return fail(VGR_ERR_INVALID_ARGUMENT, "camera ingestion arguments must be non-null");
  }
  if (count < 0 || count > INT_MAX) return fail(VGR_ERR_INVALID_ARGUMENT, "camera count must be in [0, INT_MAX]");
  if (!camera_indices && count > viewmat_count) {
    return fail(VGR_ERR_INVALID_ARGUMENT, "more world matrices than view matrices");
  }
  if (count == 0) return VGR_OK;
  vgr::world_to_opencv_kernel<<<static_cast<unsigned>((count + 255) / 256), 256, 0,
                                static_cast<cudaStream_t>(stream)>>>(
      world_matrices, camera_indices, count, viewmat_count, viewmats, invalid_index_count);
  return vgr::check_launch("world to OpenCV view matrices");
}
