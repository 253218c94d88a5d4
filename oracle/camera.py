"""ctypes wrapper of liboracle_camera.so, the CPU restatement of the camera path.

TEST INFRASTRUCTURE ONLY: used by tests/, __graft_entry__.smoke() and
bench.py's cpu_baseline leg to check or time the CUDA renderer.  See
camera_oracle.c for the reference file:line each step follows.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
_LIB: ctypes.CDLL | None = None
_p = ctypes.c_void_p
_i64 = ctypes.c_int64
_i32 = ctypes.c_int32


class _Scene(ctypes.Structure):
    _fields_ = [
        ("means", _p),
        ("covariances", _p),
        ("opacities", _p),
        ("features", _p),
        ("feature_width", _i64),
        ("semantic_ids", _p),
        ("registered_scene_ids", _p),
        ("scene_offsets", _p),
        ("scene_count", _i64),
    ]


class _Cameras(ctypes.Structure):
    _fields_ = [
        ("viewmats", _p),
        ("intrinsics", _p),
        ("env_xforms", _p),
        ("camera_scene_ids", _p),
        ("active_ids", _p),
        ("batch", _i64),
        ("active_count", _i64),
        ("widths", _p),
        ("heights", _p),
        ("tile_offsets", _p),
        ("pixel_offsets", _p),
    ]


class _Options(ctypes.Structure):
    _fields_ = [
        ("height", _i64),
        ("width", _i64),
        ("near_plane", ctypes.c_double),
        ("far_plane", ctypes.c_double),
        ("support_sigma", ctypes.c_double),
        ("covariance_epsilon", ctypes.c_double),
        ("semantic_min_alpha", ctypes.c_double),
        ("antialiased", _i32),
        ("tile_size", _i32),
        ("output_srgb", _i32),
        ("full_sensor_output", _i32),
        ("sh_degree", _i32),
        ("threads", _i32),
        ("ray_eval", _i32),
    ]


class _Stats(ctypes.Structure):
    _fields_ = [("visible", _i64), ("intersections", _i64), ("active_tiles", _i64)]


def load() -> ctypes.CDLL:
    global _LIB
    if _LIB is None:
        path = HERE / "liboracle_camera.so"
        if not path.exists():
            from . import build

            build.build()
        lib = ctypes.CDLL(str(path))
        lib.vo_render.restype = ctypes.c_int
        lib.vo_render.argtypes = [
            ctypes.POINTER(_Scene),
            ctypes.POINTER(_Cameras),
            ctypes.POINTER(_Options),
            _p,
            _p,
            _p,
            _p,
            _p,
            _i64,
            _p,
            _i64,
            ctypes.POINTER(_Stats),
        ]
        lib.vo_precompute_covariances.restype = None
        lib.vo_precompute_covariances.argtypes = [_p, _p, _i64, _p]
        lib.vo_set_margin_output.restype = None
        lib.vo_set_margin_output.argtypes = [_p]
        for name in ("vo_exp_public", "vo_log_public", "vo_srgb_public"):
            getattr(lib, name).restype = ctypes.c_float
            getattr(lib, name).argtypes = [ctypes.c_float]
        _LIB = lib
    return _LIB


def _arr(a, dtype) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a), dtype=dtype)


def _ptr(a: np.ndarray | None) -> int | None:
    return None if a is None else a.ctypes.data


def precompute_covariances(scales, rotations) -> np.ndarray:
    scales = _arr(scales, np.float32)
    rotations = _arr(rotations, np.float32)
    out = np.empty((scales.shape[0], 6), dtype=np.float32)
    load().vo_precompute_covariances(_ptr(scales), _ptr(rotations), scales.shape[0], _ptr(out))
    return out


@dataclass
class OracleResult:
    rgb: np.ndarray
    depth: np.ndarray
    alpha: np.ndarray
    semantic: np.ndarray
    visible: int
    intersections: int
    active_tiles: int
    tile_counts: np.ndarray | None
    sorted_gaussian_ids: np.ndarray | None
    margins: np.ndarray | None = None  # [..., 3] decision margins (with_margins)


def render(
    *,
    means,
    covariances,
    opacities,
    features,
    semantic_ids,
    registered_scene_ids,
    scene_offsets,
    viewmats,
    intrinsics,
    camera_scene_ids,
    height: int,
    width: int,
    env_xforms=None,
    active_ids=None,
    near_plane: float = 0.01,
    far_plane: float = 100.0,
    support_sigma: float = 3.33,
    covariance_epsilon: float = 0.3,
    semantic_min_alpha: float = 0.01,
    antialiased: bool = False,
    tile_size: int = 16,
    output_srgb: bool = False,
    sh_degree: int = -1,
    threads: int = 0,
    with_tiles: bool = False,
    ragged: dict | None = None,
    ray_gaussian_evaluation: bool = False,
    with_margins: bool = False,
) -> OracleResult:
    """Render every active camera on the CPU.  ``ragged`` may carry per-camera
    ``widths``, ``heights``, ``tile_offsets``, ``pixel_offsets`` and
    ``total_pixels``/``total_tiles`` for the mixed-resolution form.
    ``with_margins`` also returns each pixel's decision margins (relative
    distance of the closest alpha / power-cut, transmittance-stop and
    depth-order decision; see vo_set_margin_output in camera_oracle.c)."""
    means = _arr(means, np.float32)
    covariances = _arr(covariances, np.float32)
    opacities = _arr(opacities, np.float32)
    features = _arr(features, np.float32)
    semantic_ids = _arr(semantic_ids, np.int64)
    registered = _arr(registered_scene_ids, np.int64)
    offsets = _arr(scene_offsets, np.int64)
    viewmats = _arr(viewmats, np.float32)
    intrinsics = _arr(intrinsics, np.float32)
    batch = viewmats.shape[0]
    env = _arr(env_xforms if env_xforms is not None else np.tile(np.eye(4, dtype=np.float32), (batch, 1, 1)), np.float32)
    camera_scene_ids = _arr(camera_scene_ids, np.int64)
    active = None if active_ids is None else _arr(active_ids, np.int64)
    scene = _Scene(
        _ptr(means), _ptr(covariances), _ptr(opacities), _ptr(features), features.shape[1],
        _ptr(semantic_ids), _ptr(registered), _ptr(offsets), registered.shape[0],
    )
    if ragged is None:
        total_pixels = batch * height * width
        bin_size = 32 if ray_gaussian_evaluation and tile_size == 16 else tile_size
        tiles = batch * (-(-height // bin_size)) * (-(-width // bin_size))
        cams = _Cameras(
            _ptr(viewmats), _ptr(intrinsics), _ptr(env), _ptr(camera_scene_ids), _ptr(active),
            batch, 0 if active is None else active.shape[0], None, None, None, None,
        )
        keep = []
    else:
        widths = _arr(ragged["widths"], np.int32)
        heights = _arr(ragged["heights"], np.int32)
        tile_offsets = _arr(ragged["tile_offsets"], np.int64)
        pixel_offsets = _arr(ragged["pixel_offsets"], np.int64)
        keep = [widths, heights, tile_offsets, pixel_offsets]
        total_pixels = int(pixel_offsets[-1])
        tiles = int(tile_offsets[-1])
        cams = _Cameras(
            _ptr(viewmats), _ptr(intrinsics), _ptr(env), _ptr(camera_scene_ids), _ptr(active),
            batch, 0 if active is None else active.shape[0],
            _ptr(widths), _ptr(heights), _ptr(tile_offsets), _ptr(pixel_offsets),
        )
    opts = _Options(
        height, width, near_plane, far_plane, support_sigma, covariance_epsilon,
        semantic_min_alpha, int(antialiased), tile_size, int(output_srgb), 1, sh_degree, threads,
        int(ray_gaussian_evaluation),
    )
    rgb = np.zeros((total_pixels, 3), dtype=np.float32)
    depth = np.full((total_pixels,), np.inf, dtype=np.float32)
    alpha = np.zeros((total_pixels,), dtype=np.float32)
    semantic = np.full((total_pixels,), -1, dtype=np.int64)
    tile_counts = np.zeros((tiles,), dtype=np.int32) if with_tiles else None
    stats = _Stats()
    lib = load()
    margins = np.full((total_pixels, 3), np.inf, dtype=np.float32) if with_margins else None
    # First pass sizes the sorted-id list when requested.
    sorted_ids = None
    if with_tiles:
        code = lib.vo_render(scene, cams, opts, _ptr(rgb), _ptr(depth), _ptr(alpha), _ptr(semantic),
                             _ptr(tile_counts), tiles, None, 0, ctypes.byref(stats))
        if code != 0:
            raise RuntimeError("oracle render failed")
        sorted_ids = np.zeros((max(stats.intersections, 1),), dtype=np.int32)
        tile_counts[:] = 0
    lib.vo_set_margin_output(_ptr(margins))
    try:
        code = lib.vo_render(scene, cams, opts, _ptr(rgb), _ptr(depth), _ptr(alpha), _ptr(semantic),
                             _ptr(tile_counts), tiles if with_tiles else 0, _ptr(sorted_ids),
                             0 if sorted_ids is None else sorted_ids.shape[0], ctypes.byref(stats))
    finally:
        lib.vo_set_margin_output(None)
    if code != 0:
        raise RuntimeError("oracle render failed")
    del keep
    if ragged is None:
        shape = (batch, height, width)
        rgb = rgb.reshape(*shape, 3)
        depth = depth.reshape(*shape, 1)
        alpha = alpha.reshape(*shape, 1)
        semantic = semantic.reshape(*shape, 1)
        if margins is not None:
            margins = margins.reshape(*shape, 3)
    return OracleResult(
        rgb, depth, alpha, semantic, int(stats.visible), int(stats.intersections),
        int(stats.active_tiles), tile_counts,
        None if sorted_ids is None else sorted_ids[: stats.intersections],
        margins,
    )


def exp(x: float) -> float:
    return float(load().vo_exp_public(x))


def log(x: float) -> float:
    return float(load().vo_log_public(x))


def srgb(x: float) -> float:
    return float(load().vo_srgb_public(x))
