"""ctypes wrapper of liboracle_lidar.so (CPU restatement of the LiDAR oracle).

TEST INFRASTRUCTURE ONLY (tests/, __graft_entry__.smoke(), bench.py's
cpu_baseline leg).  See lidar_oracle.c for the reference lines it follows.
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
_d = ctypes.c_double


class _Config(ctypes.Structure):
    _fields_ = [
        ("near_plane", _d),
        ("far_plane", _d),
        ("support_sigma", _d),
        ("detection_threshold", _d),
        ("planarity_ratio_max", _d),
        ("min_incidence_cos", _d),
        ("cluster_abs", _d),
        ("cluster_relative", _d),
        ("fallback_reflectivity", _d),
    ]


class _Scene(ctypes.Structure):
    _fields_ = [
        ("scene_id", _i64),
        ("count", _i64),
        ("means", _p),
        ("scales", _p),
        ("rotations", _p),
        ("opacities", _p),
        ("semantics", _p),
        ("reflectivity", _p),
        ("confidence", _p),
    ]


@dataclass(frozen=True)
class LidarConfig:
    """Defaults of the reference oracle and backend (lidar_cpu_oracle.py:15-25)."""

    near_plane_m: float = 0.05
    far_plane_m: float = 200.0
    support_sigma: float = 3.0
    detection_threshold: float = 0.01
    planarity_ratio_max: float = 0.35
    min_incidence_cos: float = 0.05
    cluster_abs_m: float = 0.02
    cluster_relative: float = 0.001
    fallback_reflectivity: float = 0.5


def load() -> ctypes.CDLL:
    global _LIB
    if _LIB is None:
        path = HERE / "liboracle_lidar.so"
        if not path.exists():
            from . import build

            build.build()
        lib = ctypes.CDLL(str(path))
        lib.lo_render.restype = ctypes.c_int
        lib.lo_render.argtypes = [
            ctypes.POINTER(_Scene), _i64, _p, _i64, _p, _p, _p, _i64, _p, _i64, _i64,
            ctypes.POINTER(_Config), ctypes.c_int, _p, _p, _p, _p, _p, _p,
        ]
        _LIB = lib
    return _LIB


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64))


def render(
    scenes: dict[int, dict],
    ray_directions,
    time_offsets_ns,
    sensor_to_world,
    scene_ids,
    *,
    scene_to_world=None,
    active_sensor_ids=None,
    returns: int = 1,
    config: LidarConfig = LidarConfig(),
    threads: int = 0,
) -> dict[str, np.ndarray]:
    """Same arguments and outputs as the reference oracle's render_lidar_oracle."""
    if returns not in (1, 2):
        raise ValueError("returns must be 1 or 2.")
    dirs = _f64(ray_directions)
    norms = np.linalg.norm(dirs, axis=1)
    if not np.allclose(norms, 1.0, rtol=0.0, atol=1.0e-4):
        raise ValueError("ray_directions must be normalized.")
    sensors = _f64(sensor_to_world)
    batch = sensors.shape[0]
    rays = dirs.shape[0]
    xforms = _f64(np.repeat(np.eye(4)[None], batch, axis=0) if scene_to_world is None else scene_to_world)
    ids = np.ascontiguousarray(np.asarray(scene_ids, dtype=np.int64))
    active = None if active_sensor_ids is None else np.ascontiguousarray(np.asarray(active_sensor_ids, dtype=np.int64))
    keep = []
    native = (_Scene * max(len(scenes), 1))()
    for k, (sid, scene) in enumerate(scenes.items()):
        arrays = {
            name: _f64(scene[name]) for name in ("means", "scales", "rotations", "opacities")
        }
        rotations = arrays["rotations"]
        if not np.allclose(np.linalg.norm(rotations, axis=1), 1.0, rtol=0.0, atol=1.0e-4):
            raise ValueError("Oracle rotations must be normalized WXYZ quaternions.")
        sem = np.ascontiguousarray(np.asarray(scene["semantic_ids"], dtype=np.int64))
        refl = None if scene.get("reflectivity") is None else _f64(scene["reflectivity"])
        conf = None if scene.get("surface_confidence") is None else _f64(scene["surface_confidence"])
        keep.extend([arrays, sem, refl, conf])
        native[k] = _Scene(
            sid, arrays["means"].shape[0], arrays["means"].ctypes.data, arrays["scales"].ctypes.data,
            rotations.ctypes.data, arrays["opacities"].ctypes.data, sem.ctypes.data,
            None if refl is None else refl.ctypes.data, None if conf is None else conf.ctypes.data,
        )
    out = {
        "range_m": np.full((batch, rays, returns), np.inf),
        "position_world_m": np.zeros((batch, rays, returns, 3)),
        "intensity": np.zeros((batch, rays, returns)),
        "semantic_id": np.full((batch, rays, returns), -1, dtype=np.int64),
        "valid": np.zeros((batch, rays, returns), dtype=np.uint8),
        "return_count": np.zeros((batch, rays), dtype=np.int32),
    }
    cfg = _Config(
        config.near_plane_m, config.far_plane_m, config.support_sigma, config.detection_threshold,
        config.planarity_ratio_max, config.min_incidence_cos, config.cluster_abs_m,
        config.cluster_relative, config.fallback_reflectivity,
    )
    code = load().lo_render(
        native, len(scenes), dirs.ctypes.data, rays, sensors.ctypes.data, xforms.ctypes.data,
        ids.ctypes.data, batch, None if active is None else active.ctypes.data,
        0 if active is None else active.shape[0], returns, ctypes.byref(cfg), threads,
        out["range_m"].ctypes.data, out["position_world_m"].ctypes.data, out["intensity"].ctypes.data,
        out["semantic_id"].ctypes.data, out["valid"].ctypes.data, out["return_count"].ctypes.data,
    )
    del keep
    if code == -1:
        raise ValueError("Unregistered oracle scene ID.")
    if code != 0:
        raise RuntimeError("LiDAR oracle failed")
    out["valid"] = out["valid"].astype(bool)
    out["time_offset_ns"] = np.broadcast_to(
        np.asarray(time_offsets_ns, dtype=np.int64)[None, :, None], (batch, rays, returns)
    ).copy()
    return out
