"""ctypes declarations of the LiDAR entry points of libvgr_b200.so."""

from __future__ import annotations

import ctypes

_i64 = ctypes.c_int64
_i32 = ctypes.c_int32
_p = ctypes.c_void_p
_d = ctypes.c_double

LIDAR_COUNTERS = 12
LIDAR_DESCRIPTOR_BYTES = 112


class VgrLidarScene(ctypes.Structure):
    _fields_ = [
        ("means", _p),
        ("scales", _p),
        ("rotations", _p),
        ("opacities", _p),
        ("semantic_ids", _p),
        ("reflectivity", _p),
        ("surface_confidence", _p),
        ("count", _i64),
    ]


class VgrLidarInputs(ctypes.Structure):
    _fields_ = [
        ("ray_directions", _p),
        ("rays", _i64),
        ("time_offsets", _p),
        ("time_offsets_are_int64", _i32),
        ("sensor_to_world", _p),
        ("scene_to_world", _p),
        ("scene_ids", _p),
        ("batch", _i64),
        ("active_sensor_ids", _p),
        ("active_count", _i64),
        ("ray_order", _p),
    ]


class VgrLidarOutputs(ctypes.Structure):
    _fields_ = [
        ("range_m", _p),
        ("position_world_m", _p),
        ("intensity", _p),
        ("semantic_id", _p),
        ("valid", _p),
        ("time_offset_ns", _p),
        ("return_count", _p),
    ]


class VgrLidarOptions(ctypes.Structure):
    _fields_ = [
        ("returns", _i32),
        ("semantic_slots", _i32),
        ("near_plane_m", _d),
        ("far_plane_m", _d),
        ("support_sigma", _d),
        ("detection_threshold", _d),
        ("planarity_ratio_max", _d),
        ("min_incidence_cos", _d),
        ("cluster_abs_m", _d),
        ("cluster_relative", _d),
        ("fallback_reflectivity", _d),
        ("direction_norm_tolerance", _d),
    ]


def extra_signatures() -> list[tuple[str, object, list[object]]]:
    return [
        ("vgr_lidar_sort_temp_bytes", _i64, [_i64, _i32]),
        (
            "vgr_lidar_build_scene_lbvh",
            ctypes.c_int,
            [ctypes.POINTER(VgrLidarScene), _i32, _d, _d, _p, _i64, _p],
        ),
        ("vgr_lidar_pack_scene_descriptor", ctypes.c_int, [_p, _i64, _i64, _i64, _p, _i64, _i32, _p]),
        (
            "vgr_render_lidar",
            ctypes.c_int,
            [
                _p,
                _i64,
                ctypes.POINTER(VgrLidarInputs),
                ctypes.POINTER(VgrLidarOutputs),
                _p,
                ctypes.POINTER(VgrLidarOptions),
                _p,
            ],
        ),
    ]
