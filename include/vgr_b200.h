/*
 * vgr_b200.h -- C ABI of the B200-native batched Gaussian-splat sensor renderer.
 *
 * Every entry point takes plain pointers, sizes and a CUDA stream (as void*),
 * enqueues its work on that stream, never synchronises the host and never
 * allocates device memory.  Functions return VGR_OK (0) on success or a
 * negative VGR_ERR_* code; vgr_last_error() then returns a thread-local
 * message naming the violated contract (the same checks the reference
 * performs with TORCH_CHECK in its pybind binding).
 *
 * The entry points replace the functions the reference exports from its
 * PyTorch extension modules:
 *   src/isaacsim_gaussian_renderer/native/renderer.cpp:312-337        (camera)
 *   src/isaacsim_gaussian_renderer/native/lidar_renderer.cpp:213-216  (LiDAR)
 * Each declaration below names the reference function and the file:line of
 * its definition.  Tensor-order enums of the reference camera module are
 * at src/isaacsim_gaussian_renderer/native/renderer_cuda.cu:48-98; the
 * structs below carry the same tensors by name.
 */
#ifndef VGR_B200_H_
#define VGR_B200_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VGR_OK 0
#define VGR_ERR_INVALID_ARGUMENT (-1)
#define VGR_ERR_CUDA (-2)
#define VGR_ERR_SCRATCH_TOO_SMALL (-3)
#define VGR_ERR_UNSUPPORTED (-4)

/* Counter slots, same order as the reference COUNTER_NAMES
 * (src/isaacsim_gaussian_renderer/cuda_backend.py:22-28). */
#define VGR_COUNTER_VISIBLE 0
#define VGR_COUNTER_INTERSECTIONS 1
#define VGR_COUNTER_VISIBLE_OVERFLOW 2
#define VGR_COUNTER_INTERSECTION_OVERFLOW 3
#define VGR_COUNTER_ACTIVE_TILES 4
#define VGR_COUNTER_COUNT 5

/* One projected (camera, Gaussian) record: 48 bytes, 16-byte aligned.
 *   a = (mean_x, mean_y, conic_xx, conic_xy)
 *   b = (conic_yy, opacity, depth, bits(gaussian id))
 *   c = (red, green, blue, bits(two fp16 half-extents of the footprint box)) */
#define VGR_RECORD_BYTES 48

/* Packed scene in the reference's canonical layout (scene.py:12-33 after
 * covariance precompute, cuda_backend.py:2080-2108). */
typedef struct vgr_scene {
  const float* means;                  /* [G,3] */
  const float* covariances;            /* [G,6] upper triangle 00,01,02,11,12,22 */
  const float* opacities;              /* [G] activated */
  const float* features;               /* [G,F]; F>=3 */
  int64_t feature_width;               /* F */
  const int64_t* semantic_ids;         /* [G] */
  const int64_t* registered_scene_ids; /* [S] */
  const int64_t* scene_offsets;        /* [S+1] packed offsets */
  int64_t scene_count;                 /* S */
  int64_t gaussian_count;              /* G */
  int64_t max_scene_gaussians;         /* max_s (offsets[s+1]-offsets[s]) */
  /* Optional spatial layout (no counterpart in the reference; NULL = none).
   * gaussian_ids: packed Gaussian g is reported as gaussian_ids[g] (records,
   * depth-tie order, semantic_ids index), so a scene stored in another order
   * (vgr_scene_spatial_order) renders exactly as the original.  chunk_bounds:
   * per chunk of VGR_PROJECT_CHUNK consecutive Gaussians of a registered
   * scene, (min x, min y, min z, max covariance trace, max x, max y, max z,
   * 0) from vgr_scene_chunk_bounds; chunk_offsets[s] is scene s's first
   * chunk.  A chunk outside a camera's frustum is then not projected.
   * cluster_bounds (with chunk_bounds): the same bounds per cluster of
   * VGR_PROJECT_CLUSTER consecutive Gaussians, VGR_PROJECT_CHUNK /
   * VGR_PROJECT_CLUSTER clusters per chunk (cluster k of chunk c at row
   * c * 16 + k), from vgr_scene_cluster_bounds; a cluster outside a camera's
   * frustum inside a chunk that is not is then skipped as well. */
  const int32_t* gaussian_ids;         /* [G] or NULL */
  const float* chunk_bounds;           /* [C,8] or NULL */
  const int64_t* chunk_offsets;        /* [S+1], required with chunk_bounds */
  const float* cluster_bounds;         /* [C*16,8] or NULL */
} vgr_scene;
/* Gaussians per projection chunk (the unit of vgr_scene.chunk_bounds). */
#define VGR_PROJECT_CHUNK 512
/* Gaussians per projection cluster (the unit of vgr_scene.cluster_bounds). */
#define VGR_PROJECT_CLUSTER 32

/* Camera batch.  The plain form leaves the four per-camera resolution arrays
 * NULL and renders every camera at (height,width) of vgr_render_options.
 * The ragged form passes per-camera widths/heights plus exclusive prefixes of
 * tiles and pixels over the batch (device int64 arrays of length B+1). */
typedef struct vgr_cameras {
  const float* viewmats;           /* [B,4,4] world->OpenCV camera */
  const float* intrinsics;         /* [B,3,3] */
  const float* env_xforms;         /* [B,4,4] object->world */
  const int64_t* camera_scene_ids; /* [B] */
  const int64_t* active_camera_ids;/* [A] or NULL (all cameras) */
  int64_t batch;                   /* B */
  int64_t active_count;            /* A (== B when active_camera_ids is NULL) */
  const int32_t* widths;           /* ragged form: [B] or NULL */
  const int32_t* heights;          /* ragged form: [B] or NULL */
  const int64_t* tile_offsets;     /* ragged form: [B+1] or NULL */
  const int64_t* pixel_offsets;    /* ragged form: [B+1] or NULL */
  int64_t total_tiles;             /* ragged form: tile_offsets[B] (host copy) */
  int64_t max_tiles_per_camera;    /* ragged form: max over cameras */
} vgr_cameras;

/* Outputs, pixel-major.  Plain form: [B,H,W,C]; ragged form: [P,C] with
 * camera c at pixel_offsets[c].  depth/alpha/semantic may be NULL when
 * full_sensor_output is 0 (RGB-only contract). */
typedef struct vgr_outputs {
  float* rgb;        /* 3 channels */
  float* depth;      /* 1 channel */
  float* alpha;      /* 1 channel */
  int64_t* semantic; /* 1 channel */
} vgr_outputs;

typedef struct vgr_workspace {
  void* records;                 /* visible_capacity * VGR_RECORD_BYTES, 16-B aligned;
                                  * twice that with ray_gaussian_evaluation (the second
                                  * half holds the exact-ray extension records) */
  int64_t visible_capacity;
  uint64_t* keys_in;             /* [I] sort keys (tile<<32 | depth bits) */
  uint64_t* keys_out;            /* [I] */
  int32_t* values_in;            /* [I] visible-record indices */
  int32_t* values_out;           /* [I] */
  int64_t intersection_capacity; /* I */
  int32_t* tile_starts;          /* [T] */
  int32_t* tile_ends;            /* [T] */
  int64_t tile_capacity;         /* T >= global tile count */
  int64_t* counters;             /* [5] */
  void* scratch;                 /* vgr_render_scratch_bytes(...) bytes, 256-B aligned */
  int64_t scratch_bytes;
  /* Optional structure-of-arrays mirrors of the visible records in the
   * reference workspace layout (renderer_cuda.cu:74-80); NULL skips them. */
  float* visible_means2d;        /* [V,2] */
  float* visible_conics;         /* [V,3] */
  float* visible_depths;         /* [V] */
  float* visible_opacities;      /* [V] */
  int32_t* visible_camera_ids;   /* [V] */
  int32_t* visible_gaussian_ids; /* [V] */
  int32_t* visible_radii;        /* [V,2] */
  /* Dense mode (tile_size 1) only, else NULL: optical-thickness bounds by
   * depth bucket per 4x4-pixel cell, and the depth cutoff per 16-pixel tile. */
  float* depth_tau;              /* [B * ceil(H/4) * ceil(W/4) * VGR_DENSE_DEPTH_BUCKETS],
                                  * 16-byte aligned */
  int64_t depth_tau_capacity;    /* elements */
  int32_t* tile_cutoff;          /* [T16] */
  int64_t tile_cutoff_capacity;  /* elements */
  /* Exact-ray mode, optional mirrors in the reference workspace layout
   * (renderer_cuda.cu:96-97): per visible record the camera-space precision
   * [V,6] and (precision * mean, mean^T precision mean) [V,4]. */
  float* visible_ray_precisions;
  float* visible_ray_precision_means;
} vgr_workspace;

/* Depth buckets of dense mode's optical-thickness cutoff (16 per octave of
 * depth above near_plane). */
#define VGR_DENSE_DEPTH_BUCKETS 256
#define VGR_DENSE_CELL 4

typedef struct vgr_render_options {
  int64_t height;                 /* plain-form resolution */
  int64_t width;
  double near_plane;
  double far_plane;
  double gaussian_support_sigma;
  double covariance_epsilon;
  double semantic_min_alpha;
  int32_t antialiased;
  int32_t ray_gaussian_evaluation; /* exact ray-Gaussian evaluation (renderer_cuda.cu:795-948,
                                    * 2190-2270); records doubles; not with antialiased */
  int32_t tile_size;               /* 4, 8 or 16; 1 = dense mode (the reference's per-pixel
                                    * path): 16-pixel tiles with an optical-thickness depth
                                    * cutoff (renderer_cuda.cu:1093-1400,1658-1689) */
  int32_t output_srgb;
  int32_t deterministic;           /* accepted; ordering is always deterministic */
  int32_t full_sensor_output;
  int32_t fixed_capacity_sort;     /* accepted; the sort is always device-bounded */
  int32_t reuse_projection;        /* composite only, from the last sorted lists */
  int32_t compact_projection_cache;/* tile_size 1 only; dense mode always projects twice */
  int32_t sh_degree;               /* -1: features[0..2] are linear RGB (reference);
                                      0..3: real spherical harmonics, [G,(d+1)^2*3] */
  int32_t sorted_buffer_hint;      /* reuse_projection: 1 if sorted data lives in *_out */
  /* Optional timing hook (no counterpart in the reference): when non-NULL,
   * stage_events[i] (cudaEvent_t) is recorded on the stream at stage
   * boundary i: 0 start, 1 after camera setup, 2 after projection+emission,
   * 3 after the sort histogram, 4 after the radix passes, 5 after tile
   * ranges, 6 after compositing.  stage_event_count must be 7. */
  void* const* stage_events;
  int32_t stage_event_count;
  /* Compositor launch (no counterpart in the reference): 0 = one CTA per
   * (camera, tile); 1 = a resident grid taking (camera, tile) work items from
   * a device queue. */
  int32_t persistent_compositor;
  /* Compositor CTA shape (no counterpart in the reference; 8-, 16- and
   * 32-pixel tiles of the screen-space forward path): 0 = two pixels per
   * thread at the tuned occupancy; 1 = one pixel per thread (8x4-pixel warp
   * blocks, twice the threads); 2 = two pixels per thread at half
   * occupancy.  Every shape renders the same bits. */
  int32_t composite_shape;
} vgr_render_options;

#define VGR_STAGE_EVENTS 7

/* Library identity. */
const char* vgr_version(void);
/* Number of kernels this library has launched in this process (all threads).
 * No counterpart in the reference; used to attribute launches in benchmarks. */
int64_t vgr_kernel_launch_count(void);
/* VGR_PROJECT_CHUNK of the loaded library: the number of Gaussians per row of
 * vgr_scene.chunk_bounds (a host that sizes the bounds at run time asks the
 * library rather than its own copy of the header). */
int64_t vgr_project_chunk(void);
/* Thread-local message of the last failing call on this thread. */
const char* vgr_last_error(void);

/* Scratch bytes vgr_render needs for a given intersection capacity, projection
 * task bound (active cameras * max scene Gaussians), global tile count and
 * active-camera bound.  The size depends only on the active-camera bound
 * (per-camera plans and projection constants) and a constant part;
 * max_projection_tasks and global_tiles are validated and otherwise ignored
 * (accepted for interface stability).  No counterpart in the reference: the
 * reference sizes CUB temporary storage through the two functions below. */
int64_t vgr_render_scratch_bytes(int64_t intersection_capacity,
                                 int64_t max_projection_tasks,
                                 int64_t global_tiles,
                                 int64_t max_active_cameras);

/* Replaces sort_temp_bytes (renderer.cpp:76-81, renderer_cuda.cu:2463-2508).
 * Returns the scratch bytes of the deterministic path for num_items keys and
 * num_segments tiles, or a negative error code. */
int64_t vgr_sort_temp_bytes(int64_t num_items, int64_t num_segments);

/* Replaces radix_sort_double_buffer_temp_bytes (renderer.cpp:83-90,
 * renderer_cuda.cu:2510-2534). */
int64_t vgr_radix_sort_double_buffer_temp_bytes(int64_t num_items,
                                                int64_t num_segments);

/* Replaces precompute_covariances (renderer.cpp:92-131,
 * renderer_cuda.cu:492-540,2374-2395): Sigma = R S S^T R^T from WXYZ
 * quaternions and activated scales, upper triangle [G,6]. */
int vgr_precompute_covariances(const float* scales, const float* rotations,
                               int64_t gaussian_count, float* covariances,
                               void* stream);

/* Replaces prepare_chunked_active_ids (renderer.cpp:133-181,
 * renderer_cuda.cu:2307-2338,2397-2444). */
int vgr_prepare_chunked_active_ids(const int64_t* active_camera_ids,
                                   int64_t active_count, int32_t* active_mask,
                                   int64_t active_mask_capacity,
                                   int64_t* chunk_active_ids,
                                   int64_t chunk_rows, int64_t chunk_columns,
                                   int64_t logical_batch,
                                   int64_t physical_batch, void* stream);

/* Replaces aggregate_chunk_counters (renderer.cpp:183-212,
 * renderer_cuda.cu:2340-2360,2446-2461). */
int vgr_aggregate_chunk_counters(const int64_t* chunk_counters,
                                 int64_t chunk_rows, int64_t chunk_stride,
                                 int64_t* counters,
                                 int64_t* physical_capacity_counters,
                                 int64_t chunk_count, void* stream);

/* Replaces render (renderer.cpp:214-310, renderer_cuda.cu:2536-3456):
 * projection + ordered compaction + tile emission, device-bounded stable LSD
 * radix sort of (tile, depth) keys, tile ranges and the fused
 * RGB/depth/alpha/semantic compositor.  *sorted_buffer_selector receives 1
 * when keys_out/values_out hold the sorted lists and 0 when keys_in/values_in
 * do (the reference's CUB DoubleBuffer selector). */
int vgr_render(const vgr_scene* scene, const vgr_cameras* cameras,
               const vgr_outputs* outputs, const vgr_workspace* workspace,
               const vgr_render_options* options, void* stream,
               int64_t* sorted_buffer_selector);

/* Size of the library-owned device array used by vgr_render_static_scratch. */
#define VGR_STATIC_SCRATCH_BYTES (16ll << 20)

/* vgr_render for callers that must not allocate device memory on their
 * render path (a plug-in whose host owns every device allocation through its
 * own pool, a real-time loop that cannot afford allocator latency, code being
 * recorded into a CUDA graph).  It has no counterpart in the reference.  The
 * caller passes inputs, outputs and the record/key/value/range/counter
 * workspace exactly as for vgr_render; workspace->scratch and scratch_bytes
 * are ignored and a VGR_STATIC_SCRATCH_BYTES array inside the library is used
 * instead (every GPU that loads the library keeps it until exit).  The
 * scratch grows with the active cameras (176 bytes each, plus about 9 KB),
 * not with the scene or the intersections: a render of more than
 * vgr_static_scratch_max_cameras() active cameras (95,275) fails with
 * VGR_ERR_SCRATCH_TOO_SMALL before anything is launched.  reuse_projection is
 * refused (VGR_ERR_INVALID_ARGUMENT): the shared array may hold another
 * call's camera plans.  Nothing is allocated.  All calls share the array:
 * calls ordered on one stream are fine, calls that overlap on the GPU race.
 * The first call on a device looks the array's address up while that device
 * is current and caches it for the process; make it before any stream
 * capture.  The address belongs to the device's primary context: do not call
 * this after cudaDeviceReset, or from a driver-API context of one's own. */
int vgr_render_static_scratch(const vgr_scene* scene, const vgr_cameras* cameras,
                              const vgr_outputs* outputs,
                              const vgr_workspace* workspace,
                              const vgr_render_options* options, void* stream,
                              int64_t* sorted_buffer_selector);
/* Largest active-camera count whose scratch fits in the static array of
 * vgr_render_static_scratch (no counterpart in the reference). */
int64_t vgr_static_scratch_max_cameras(void);

/* Spatial layout of a scene (no counterpart in the reference).  Temp bytes
 * of vgr_scene_spatial_order for a scene of gaussian_count Gaussians. */
int64_t vgr_scene_spatial_order_temp_bytes(int64_t gaussian_count);
/* order[i] = index of the i-th Gaussian in Morton order of the means (30-bit
 * keys over the means' bounding box, stable).  Storing a scene in this order
 * makes projection chunks spatially compact. */
int vgr_scene_spatial_order(const float* means, int64_t gaussian_count, int32_t* order,
                            void* temp, int64_t temp_bytes, void* stream);
/* Bounds of each chunk of VGR_PROJECT_CHUNK consecutive Gaussians of one
 * scene: bounds[c*8 .. c*8+7] = (min x, min y, min z, max covariance trace,
 * max x, max y, max z, 0), ceil(gaussian_count / VGR_PROJECT_CHUNK) chunks. */
int vgr_scene_chunk_bounds(const float* means, const float* covariances,
                           int64_t gaussian_count, float* bounds, void* stream);
/* The same bounds per cluster of VGR_PROJECT_CLUSTER consecutive Gaussians
 * of one scene: ceil(gaussian_count / VGR_PROJECT_CHUNK) * 16 rows of 8
 * floats (clusters past the end of the scene hold an empty box). */
int vgr_scene_cluster_bounds(const float* means, const float* covariances,
                             int64_t gaussian_count, float* bounds, void* stream);
/* ---------------------------------------------------------------- ingestion */
/* Scalar types of PLY properties (PLY names: char uchar short ushort int uint
 * float double, and int64 for a semantic_id written by 64-bit tools). */
#define VGR_PLY_INT8 0
#define VGR_PLY_UINT8 1
#define VGR_PLY_INT16 2
#define VGR_PLY_UINT16 3
#define VGR_PLY_INT32 4
#define VGR_PLY_UINT32 5
#define VGR_PLY_INT64 6
#define VGR_PLY_FLOAT32 7
#define VGR_PLY_FLOAT64 8
/* Property roles (index into vgr_ply_layout.offsets/types). */
#define VGR_PLY_X 0
#define VGR_PLY_SCALE0 3
#define VGR_PLY_ROT0 6
#define VGR_PLY_OPACITY 10
#define VGR_PLY_DC0 11
#define VGR_PLY_SEMANTIC 14
#define VGR_PLY_REST0 15
#define VGR_PLY_MAX_PROPERTIES 64
/* Byte layout of one packed vertex row of an INRIA 3DGS PLY body: x y z,
 * scale_0..2, rot_0..3 (WXYZ), opacity, f_dc_0..2, semantic_id (optional),
 * then f_rest_0..f_rest_{rest_count-1}. */
typedef struct vgr_ply_layout {
  int64_t row_bytes;
  int32_t offsets[VGR_PLY_MAX_PROPERTIES];
  int32_t types[VGR_PLY_MAX_PROPERTIES];
  int32_t rest_count;  /* multiple of 3 */
  int32_t has_semantic;
} vgr_ply_layout;
/* Replaces load_ply_to_gaussians + canonicalize_3dgs_scene
 * (ply_loader.py:52-135) after the host has read the header and copied the
 * vertex rows to the device: means [G,3], scales = exp [G,3], rotations =
 * q / |q| (identity when |q| <= float32 eps) [G,4], opacities = sigmoid [G],
 * features [G,F] = (clamp(0.5 + SH_C0 dc, 0, 1), f_rest coefficient-major,
 * zero padding), semantic_ids [G] (0 without a semantic_id property). */
int vgr_ply_canonicalize(const void* vertex_rows, int64_t count, const vgr_ply_layout* layout,
                         float* means, float* scales, float* rotations, float* opacities,
                         float* features, int64_t feature_width, int64_t* semantic_ids,
                         void* stream);
/* Replaces the Warp kernel fabric_world_to_opencv_viewmats
 * (fabric_camera_kernels.py:8-49): USD row-vector world matrices [N,4,4]
 * float64 -> OpenCV world->camera view matrices, camera i written to row
 * camera_indices[i] (or i when NULL) of viewmats [viewmat_count,4,4];
 * out-of-range indices are skipped and counted in *invalid_index_count
 * (device int32, caller-zeroed). */
int vgr_world_to_opencv_viewmats(const double* world_matrices, const int32_t* camera_indices,
                                 int64_t count, float* viewmats, int64_t viewmat_count,
                                 int32_t* invalid_index_count, void* stream);
/* Replaces composite_gaussian_and_mesh (hybrid_compositor.py:21-128): the
 * depth-ordered straight-alpha composite of a Gaussian render and a mesh
 * render, all [P] / [P,3] float32 pixel-major; mesh_in_front is [P] uint8.
 * Same validity rules (alpha > min_alpha, finite alpha and depth), result
 * bit-identical to the reference's float32 tensor expression. */
int vgr_composite_gaussian_and_mesh(const float* gaussian_rgb, const float* gaussian_alpha,
                                    const float* gaussian_depth, const float* mesh_rgb,
                                    const float* mesh_alpha, const float* mesh_depth,
                                    int64_t pixels, double min_alpha, double depth_epsilon,
                                    float* rgb, float* alpha, float* depth,
                                    uint8_t* mesh_in_front, void* stream);
/* ----------------------------------------------------- differentiable form */
/* Training form of the camera path: the forward above plus hand-written
 * backward kernels for the compositor and the projection.  No counterpart in
 * the reference, which renders forward only and measures gradients through
 * gsplat's rasterization (benchmarks/compare_custom_gsplat.py:1163-1203).
 * Parameters are the raw optimisation variables; the forward applies
 * scale = exp(log_scale), q / |q| and opacity = sigmoid(logit). */
typedef struct vgr_train_params {
  const float* log_scales;     /* [G,3] */
  const float* rotations;      /* [G,4] WXYZ, any norm */
  const float* opacity_logits; /* [G] */
} vgr_train_params;
/* Per-frame state the forward leaves for the backward.  P = output pixels,
 * A = active cameras. */
typedef struct vgr_train_state {
  float* final_transmittance;  /* [P] */
  int32_t* last_position;      /* [P] sorted position one past the last blended record */
  int32_t* record_map;         /* [A, max_scene_gaussians] record of (camera, Gaussian) or -1 */
  int64_t record_map_capacity; /* elements */
  void* record_grads;          /* visible_capacity * VGR_RECORD_BYTES, 16-byte aligned */
} vgr_train_state;
/* Gradients of the loss with respect to the forward outputs (pixel-major,
 * same layout as vgr_outputs). */
typedef struct vgr_output_grads {
  const float* rgb;   /* [P,3] */
  const float* depth; /* [P] or NULL */
  const float* alpha; /* [P] or NULL */
} vgr_output_grads;
/* Gradients with respect to the parameters; every element is written. */
typedef struct vgr_param_grads {
  float* means;          /* [G,3] */
  float* log_scales;     /* [G,3] */
  float* rotations;      /* [G,4] */
  float* opacity_logits; /* [G] */
  float* features;       /* [G,F] */
} vgr_param_grads;
/* Activation: covariances [G,6] (as vgr_precompute_covariances with
 * exp(log_scales)) and opacities [G] = sigmoid(opacity_logits), for the
 * scene passed to vgr_render_train. */
int vgr_train_activate(const vgr_train_params* params, int64_t gaussian_count,
                       float* covariances, float* opacities, void* stream);
/* vgr_render that also fills the training state.  Requires
 * full_sensor_output = 1, output_srgb = 0, antialiased = 0 and
 * reuse_projection = 0. */
int vgr_render_train(const vgr_scene* scene, const vgr_cameras* cameras,
                     const vgr_outputs* outputs, const vgr_workspace* workspace,
                     const vgr_render_options* options, const vgr_train_state* state,
                     void* stream, int64_t* sorted_buffer_selector);
/* Backward of the last vgr_render_train with the same arguments (workspace,
 * scratch and state untouched since): compositor backward into per-record
 * gradients, then one pass per Gaussian over the cameras that saw it through
 * the projection, the colour model and the activations. */
int vgr_render_backward(const vgr_scene* scene, const vgr_train_params* params,
                        const vgr_cameras* cameras, const vgr_outputs* outputs,
                        const vgr_workspace* workspace, const vgr_render_options* options,
                        const vgr_train_state* state, const vgr_output_grads* grads,
                        const vgr_param_grads* param_grads, void* stream);
/* Training loss of the differentiable form's benchmark and trainers:
 * L = mean((rgb - target_rgb)^2) + depth_weight * sum(|depth - target_depth|)
 * / pixels, the depth term over pixels where both depths are finite.  Writes
 * loss[0] and the gradients dL/drgb [P,3] and dL/ddepth [P] in one pass. */
int vgr_photometric_loss(const float* rgb, const float* target_rgb, const float* depth,
                         const float* target_depth, int64_t pixels, double depth_weight,
                         float* loss, float* grad_rgb, float* grad_depth, void* stream);
/* ------------------------------------------------------------------ LiDAR */

/* Caller-owned Gaussian LiDAR scene (lidar_scene.py:13-96): WXYZ rotations,
 * activated scales/opacity; reflectivity and surface_confidence may be NULL
 * (constant fallback reflectivity, confidence 1). */
typedef struct vgr_lidar_scene {
  const float* means;              /* [G,3] */
  const float* scales;             /* [G,3] */
  const float* rotations;          /* [G,4] WXYZ */
  const float* opacities;          /* [G] */
  const int64_t* semantic_ids;     /* [G] */
  const float* reflectivity;       /* [G] or NULL */
  const float* surface_confidence; /* [G] or NULL */
  int64_t count;                   /* G */
} vgr_lidar_scene;

/* Shared sensor-local rays against per-sensor scenes
 * (lidar_renderer.cpp:133-210 inputs[6]). */
/* A trace order for vgr_lidar_inputs.ray_order (no counterpart in the
 * reference): the rays sorted by the 30-bit Hilbert-curve position of their
 * direction's azimuth and elevation on one angular grid, so 32 consecutive
 * entries are a compact patch of directions.  temp: vgr_lidar_ray_order_temp_bytes(rays)
 * bytes, 256-byte aligned.  Compute it once per direction set. */
int64_t vgr_lidar_ray_order_temp_bytes(int64_t rays);
int vgr_lidar_ray_order(const float* ray_directions, int64_t rays, int32_t* order, void* temp,
                        int64_t temp_bytes, void* stream);

typedef struct vgr_lidar_inputs {
  const float* ray_directions;      /* [R,3] unit, sensor frame */
  int64_t rays;                     /* R */
  const void* time_offsets;         /* [R] int32 or int64 */
  int32_t time_offsets_are_int64;
  const float* sensor_to_world;     /* [B,4,4] */
  const float* scene_to_world;      /* [B,4,4] */
  const int64_t* scene_ids;         /* [B] */
  int64_t batch;                    /* B */
  const int64_t* active_sensor_ids; /* [A] strictly increasing, or NULL (all) */
  int64_t active_count;
  /* Optional (no counterpart in the reference; NULL = ray order): a
   * permutation of 0..R-1 in which the rays are traced, 32 consecutive
   * entries per warp.  Rays whose directions are close share most of their
   * hierarchy walk, so an order that groups them (vgr_lidar_ray_order)
   * traces faster; outputs stay indexed by ray.  An entry outside 0..R-1 is counted as an
   * invalid direction and traces nothing. */
  const int32_t* ray_order;         /* [R] or NULL */
} vgr_lidar_inputs;

/* outputs[7] of the reference: every element is rewritten each call. */
typedef struct vgr_lidar_outputs {
  float* range_m;            /* [B,R,K] (+inf when no return) */
  float* position_world_m;   /* [B,R,K,3] */
  float* intensity;          /* [B,R,K] */
  int64_t* semantic_id;      /* [B,R,K] (-1 when no return) */
  uint8_t* valid;            /* [B,R,K] bool */
  int64_t* time_offset_ns;   /* [B,R,K] */
  int32_t* return_count;     /* [B,R] */
} vgr_lidar_outputs;

typedef struct vgr_lidar_options {
  int32_t returns;           /* 1 or 2 */
  int32_t semantic_slots;    /* 1..32 */
  double near_plane_m;
  double far_plane_m;
  double support_sigma;
  double detection_threshold;
  double planarity_ratio_max;
  double min_incidence_cos;
  double cluster_abs_m;
  double cluster_relative;
  double fallback_reflectivity;
  double direction_norm_tolerance;
} vgr_lidar_options;

/* Counter slots, same order as the reference LIDAR_COUNTER_NAMES
 * (cuda_lidar_backend.py:19-32). */
#define VGR_LIDAR_COUNTERS 12
/* One scene descriptor occupies at most one reference [S,14] int64 row. */
#define VGR_LIDAR_DESCRIPTOR_BYTES 112

/* Replaces sort_temp_bytes (lidar_renderer.cpp:62-65,
 * lidar_renderer_cuda.cu:853-868): bytes of the per-scene acceleration
 * buffer (surfel records, LBVH nodes and the build's sort scratch). */
int64_t vgr_lidar_sort_temp_bytes(int64_t num_items, int32_t packet_size);

/* Replaces build_scene_lbvh (lidar_renderer.cpp:67-108,
 * lidar_renderer_cuda.cu:870-929): Morton sort of the planar surfels, packet
 * leaves, Karras radix tree and bottom-up box refit, into accel. */
int vgr_lidar_build_scene_lbvh(const vgr_lidar_scene* scene, int32_t packet_size,
                               double support_sigma, double planarity_ratio_max,
                               void* accel, int64_t accel_bytes, void* stream);

/* Replaces pack_scene_descriptor (lidar_renderer.cpp:110-131,
 * lidar_renderer_cuda.cu:931-959): writes descriptor slot `slot` of a device
 * table of VGR_LIDAR_DESCRIPTOR_BYTES-byte rows. */
int vgr_lidar_pack_scene_descriptor(void* descriptors, int64_t descriptor_capacity,
                                    int64_t slot, int64_t scene_id, const void* accel,
                                    int64_t gaussian_count, int32_t packet_size,
                                    void* stream);

/* Replaces render_lidar (lidar_renderer.cpp:133-210,
 * lidar_renderer_cuda.cu:961-1051): no-hit clear, first-return tracing of
 * every (active sensor, ray), device counters[VGR_LIDAR_COUNTERS]. */
int vgr_render_lidar(const void* descriptors, int64_t scene_count,
                     const vgr_lidar_inputs* inputs, const vgr_lidar_outputs* outputs,
                     int64_t* counters, const vgr_lidar_options* options, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* VGR_B200_H_ */
