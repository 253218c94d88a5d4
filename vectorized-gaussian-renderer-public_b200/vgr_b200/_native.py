"""ctypes binding of libvgr_b200.so (the C ABI declared in include/vgr_b200.h).

The library is built in-tree by ``csrc/build.py`` into ``vgr_b200/_lib``.
Loading fails loudly when it is missing: there is no CPU fallback for any
entry point.  Functions here take raw pointers; the torch-facing layers
(``native_module``, ``cuda_backend``) validate tensors first.
"""

from __future__ import annotations

import ctypes
import os
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "_lib" / "libvgr_b200.so"

VGR_OK = 0
VGR_ERR_INVALID_ARGUMENT = -1
VGR_ERR_CUDA = -2
VGR_ERR_SCRATCH_TOO_SMALL = -3
VGR_ERR_UNSUPPORTED = -4
RECORD_BYTES = 48
PROJECT_CHUNK = 512
PROJECT_CLUSTER = 32
DENSE_DEPTH_BUCKETS = 256
DENSE_CELL = 4
STAGE_EVENTS = 7

_c_i64 = ctypes.c_int64
_c_i32 = ctypes.c_int32
_c_p = ctypes.c_void_p


class VgrScene(ctypes.Structure):
    _fields_ = [
        ("means", _c_p),
        ("covariances", _c_p),
        ("opacities", _c_p),
        ("features", _c_p),
        ("feature_width", _c_i64),
        ("semantic_ids", _c_p),
        ("registered_scene_ids", _c_p),
        ("scene_offsets", _c_p),
        ("scene_count", _c_i64),
        ("gaussian_count", _c_i64),
        ("max_scene_gaussians", _c_i64),
        ("gaussian_ids", _c_p),
        ("chunk_bounds", _c_p),
        ("chunk_offsets", _c_p),
        ("cluster_bounds", _c_p),
    ]


class VgrCameras(ctypes.Structure):
    _fields_ = [
        ("viewmats", _c_p),
        ("intrinsics", _c_p),
        ("env_xforms", _c_p),
        ("camera_scene_ids", _c_p),
        ("active_camera_ids", _c_p),
        ("batch", _c_i64),
        ("active_count", _c_i64),
        ("widths", _c_p),
        ("heights", _c_p),
        ("tile_offsets", _c_p),
        ("pixel_offsets", _c_p),
        ("total_tiles", _c_i64),
        ("max_tiles_per_camera", _c_i64),
    ]


class VgrOutputs(ctypes.Structure):
    _fields_ = [("rgb", _c_p), ("depth", _c_p), ("alpha", _c_p), ("semantic", _c_p)]


class VgrWorkspace(ctypes.Structure):
    _fields_ = [
        ("records", _c_p),
        ("visible_capacity", _c_i64),
        ("keys_in", _c_p),
        ("keys_out", _c_p),
        ("values_in", _c_p),
        ("values_out", _c_p),
        ("intersection_capacity", _c_i64),
        ("tile_starts", _c_p),
        ("tile_ends", _c_p),
        ("tile_capacity", _c_i64),
        ("counters", _c_p),
        ("scratch", _c_p),
        ("scratch_bytes", _c_i64),
        ("visible_means2d", _c_p),
        ("visible_conics", _c_p),
        ("visible_depths", _c_p),
        ("visible_opacities", _c_p),
        ("visible_camera_ids", _c_p),
        ("visible_gaussian_ids", _c_p),
        ("visible_radii", _c_p),
        ("depth_tau", _c_p),
        ("depth_tau_capacity", _c_i64),
        ("tile_cutoff", _c_p),
        ("tile_cutoff_capacity", _c_i64),
        ("visible_ray_precisions", _c_p),
        ("visible_ray_precision_means", _c_p),
    ]


class VgrRenderOptions(ctypes.Structure):
    _fields_ = [
        ("height", _c_i64),
        ("width", _c_i64),
        ("near_plane", ctypes.c_double),
        ("far_plane", ctypes.c_double),
        ("gaussian_support_sigma", ctypes.c_double),
        ("covariance_epsilon", ctypes.c_double),
        ("semantic_min_alpha", ctypes.c_double),
        ("antialiased", _c_i32),
        ("ray_gaussian_evaluation", _c_i32),
        ("tile_size", _c_i32),
        ("output_srgb", _c_i32),
        ("deterministic", _c_i32),
        ("full_sensor_output", _c_i32),
        ("fixed_capacity_sort", _c_i32),
        ("reuse_projection", _c_i32),
        ("compact_projection_cache", _c_i32),
        ("sh_degree", _c_i32),
        ("sorted_buffer_hint", _c_i32),
        ("stage_events", ctypes.POINTER(_c_p)),
        ("stage_event_count", _c_i32),
        ("persistent_compositor", _c_i32),
        ("composite_shape", _c_i32),
    ]


class VgrTrainParams(ctypes.Structure):
    _fields_ = [("log_scales", _c_p), ("rotations", _c_p), ("opacity_logits", _c_p)]


class VgrTrainState(ctypes.Structure):
    _fields_ = [
        ("final_transmittance", _c_p),
        ("last_position", _c_p),
        ("record_map", _c_p),
        ("record_map_capacity", _c_i64),
        ("record_grads", _c_p),
    ]


class VgrOutputGrads(ctypes.Structure):
    _fields_ = [("rgb", _c_p), ("depth", _c_p), ("alpha", _c_p)]


class VgrParamGrads(ctypes.Structure):
    _fields_ = [
        ("means", _c_p),
        ("log_scales", _c_p),
        ("rotations", _c_p),
        ("opacity_logits", _c_p),
        ("features", _c_p),
    ]


PLY_MAX_PROPERTIES = 64


class VgrPlyLayout(ctypes.Structure):
    _fields_ = [
        ("row_bytes", _c_i64),
        ("offsets", _c_i32 * PLY_MAX_PROPERTIES),
        ("types", _c_i32 * PLY_MAX_PROPERTIES),
        ("rest_count", _c_i32),
        ("has_semantic", _c_i32),
    ]


# (name, restype, argtypes) of every exported entry point, in header order.
CAMERA_SIGNATURES: list[tuple[str, object, list[object]]] = [
    ("vgr_version", ctypes.c_char_p, []),
    ("vgr_kernel_launch_count", _c_i64, []),
    ("vgr_project_chunk", _c_i64, []),
    ("vgr_last_error", ctypes.c_char_p, []),
    ("vgr_render_scratch_bytes", _c_i64, [_c_i64, _c_i64, _c_i64, _c_i64]),
    ("vgr_sort_temp_bytes", _c_i64, [_c_i64, _c_i64]),
    ("vgr_radix_sort_double_buffer_temp_bytes", _c_i64, [_c_i64, _c_i64]),
    ("vgr_precompute_covariances", ctypes.c_int, [_c_p, _c_p, _c_i64, _c_p, _c_p]),
    (
        "vgr_prepare_chunked_active_ids",
        ctypes.c_int,
        [_c_p, _c_i64, _c_p, _c_i64, _c_p, _c_i64, _c_i64, _c_i64, _c_i64, _c_p],
    ),
    (
        "vgr_aggregate_chunk_counters",
        ctypes.c_int,
        [_c_p, _c_i64, _c_i64, _c_p, _c_p, _c_i64, _c_p],
    ),
    (
        "vgr_render",
        ctypes.c_int,
        [
            ctypes.POINTER(VgrScene),
            ctypes.POINTER(VgrCameras),
            ctypes.POINTER(VgrOutputs),
            ctypes.POINTER(VgrWorkspace),
            ctypes.POINTER(VgrRenderOptions),
            _c_p,
            ctypes.POINTER(_c_i64),
        ],
    ),
    (
        "vgr_render_static_scratch",
        ctypes.c_int,
        [
            ctypes.POINTER(VgrScene),
            ctypes.POINTER(VgrCameras),
            ctypes.POINTER(VgrOutputs),
            ctypes.POINTER(VgrWorkspace),
            ctypes.POINTER(VgrRenderOptions),
            _c_p,
            ctypes.POINTER(_c_i64),
        ],
    ),
    ("vgr_static_scratch_max_cameras", _c_i64, []),
    (
        "vgr_ply_canonicalize",
        ctypes.c_int,
        [_c_p, _c_i64, ctypes.POINTER(VgrPlyLayout), _c_p, _c_p, _c_p, _c_p, _c_p, _c_i64, _c_p, _c_p],
    ),
    ("vgr_world_to_opencv_viewmats", ctypes.c_int, [_c_p, _c_p, _c_i64, _c_p, _c_i64, _c_p, _c_p]),
    (
        "vgr_composite_gaussian_and_mesh",
        ctypes.c_int,
        [_c_p, _c_p, _c_p, _c_p, _c_p, _c_p, _c_i64, ctypes.c_double, ctypes.c_double, _c_p, _c_p, _c_p, _c_p, _c_p],
    ),
    ("vgr_scene_spatial_order_temp_bytes", _c_i64, [_c_i64]),
    ("vgr_scene_spatial_order", ctypes.c_int, [_c_p, _c_i64, _c_p, _c_p, _c_i64, _c_p]),
    ("vgr_scene_chunk_bounds", ctypes.c_int, [_c_p, _c_p, _c_i64, _c_p, _c_p]),
    ("vgr_scene_cluster_bounds", ctypes.c_int, [_c_p, _c_p, _c_i64, _c_p, _c_p]),
    ("vgr_lidar_ray_order_temp_bytes", _c_i64, [_c_i64]),
    ("vgr_lidar_ray_order", ctypes.c_int, [_c_p, _c_i64, _c_p, _c_p, _c_i64, _c_p]),
    (
        "vgr_train_activate",
        ctypes.c_int,
        [ctypes.POINTER(VgrTrainParams), _c_i64, _c_p, _c_p, _c_p],
    ),
    (
        "vgr_render_train",
        ctypes.c_int,
        [
            ctypes.POINTER(VgrScene),
            ctypes.POINTER(VgrCameras),
            ctypes.POINTER(VgrOutputs),
            ctypes.POINTER(VgrWorkspace),
            ctypes.POINTER(VgrRenderOptions),
            ctypes.POINTER(VgrTrainState),
            _c_p,
            ctypes.POINTER(_c_i64),
        ],
    ),
    (
        "vgr_photometric_loss",
        ctypes.c_int,
        [_c_p, _c_p, _c_p, _c_p, _c_i64, ctypes.c_double, _c_p, _c_p, _c_p, _c_p],
    ),
    (
        "vgr_render_backward",
        ctypes.c_int,
        [
            ctypes.POINTER(VgrScene),
            ctypes.POINTER(VgrTrainParams),
            ctypes.POINTER(VgrCameras),
            ctypes.POINTER(VgrOutputs),
            ctypes.POINTER(VgrWorkspace),
            ctypes.POINTER(VgrRenderOptions),
            ctypes.POINTER(VgrTrainState),
            ctypes.POINTER(VgrOutputGrads),
            ctypes.POINTER(VgrParamGrads),
            _c_p,
        ],
    ),
]

_LIB: ctypes.CDLL | None = None


def library_path() -> Path:
    override = os.environ.get("VGR_B200_LIBRARY")
    return Path(override) if override else LIB_PATH


def load_library() -> ctypes.CDLL:
    """Load and type the shared library once; raise if it was never built."""
    global _LIB
    if _LIB is not None:
        return _LIB
    path = library_path()
    if not path.exists():
        raise RuntimeError(
            f"libvgr_b200.so is not built ({path}); run "
            "`python vectorized-gaussian-renderer-public_b200/csrc/build.py` "
            "(the renderer has no CPU fallback)."
        )
    lib = ctypes.CDLL(str(path))
    from . import _native_signatures

    for name, restype, argtypes in CAMERA_SIGNATURES + _native_signatures.extra_signatures():
        fn = getattr(lib, name)
        fn.restype = restype
        fn.argtypes = argtypes
    _LIB = lib
    return lib


def last_error() -> str:
    raw = load_library().vgr_last_error()
    return raw.decode("utf-8", "replace") if raw else ""


def check(code: int, what: str) -> None:
    """Raise RuntimeError (TORCH_CHECK's exception type) for a failing call."""
    if code != VGR_OK:
        raise RuntimeError(f"{what}: {last_error()}")


def check_size(value: int, what: str) -> int:
    if value < 0:
        raise RuntimeError(f"{what}: {last_error()}")
    return int(value)
