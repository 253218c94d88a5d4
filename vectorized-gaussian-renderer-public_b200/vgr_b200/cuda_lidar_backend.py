"""B200 Gaussian-LiDAR backend behind the reference's ``GaussianLidarBackend`` seam.

Drop-in for src/isaacsim_gaussian_renderer/cuda_lidar_backend.py:55-385: the
same constructor options and validation, one acceleration structure per
registered scene (rebuilt on explicit revision), a device descriptor table,
current-stream submission without host synchronisation, the
LIDAR_COUNTER_NAMES device counters and ``check_errors``.  Underneath, each
scene's acceleration is one buffer holding the Morton-ordered planar surfel
records and a Karras LBVH with child boxes in the parents (see
csrc/lidar.cu), built and traced through the C ABI of libvgr_b200.so.
"""

from __future__ import annotations

from collections import OrderedDict
from dataclasses import dataclass
from typing import Any

import torch

from . import _native
from ._native_signatures import (
    LIDAR_COUNTERS,
    LIDAR_DESCRIPTOR_BYTES,
    VgrLidarInputs,
    VgrLidarOptions,
    VgrLidarOutputs,
    VgrLidarScene,
)
from .lidar_backend import LidarRenderRequest
from .lidar_scene import GaussianLidarScene

LIDAR_COUNTER_NAMES = (
    "calls_started",
    "calls_completed",
    "rays_traced",
    "node_visits",
    "leaf_tests",
    "candidates",
    "returns",
    "stack_overflow",
    "semantic_overflow",
    "invalid_directions",
    "invalid_scene_ids",
    "invalid_active_sensor_ids",
)
assert len(LIDAR_COUNTER_NAMES) == LIDAR_COUNTERS


class LidarTraversalError(RuntimeError):
    """Raised by an explicit post-submit device-counter check."""


@dataclass
class _SceneAcceleration:
    scene: GaussianLidarScene
    accel: torch.Tensor

    @property
    def bvh_bytes(self) -> int:
        return int(self.accel.numel())


class RayOrder:
    """Trace order of a ray-direction tensor: ``vgr_lidar_ray_order``, a Hilbert
    order of the directions' azimuth and elevation, so the 32 rays a warp
    traces together are a compact patch of directions and share most of their
    hierarchy walk.  Recomputed only when the tensor's storage, length or
    version changes."""

    def __init__(self) -> None:
        self._key: tuple | None = None
        self._order: torch.Tensor | None = None
        self._temp: torch.Tensor | None = None

    def __call__(self, directions: torch.Tensor) -> torch.Tensor:
        key = (directions.device, directions.data_ptr(), directions.shape[0], directions._version)
        if key != self._key or self._order is None:
            rays = directions.shape[0]
            lib = _native.load_library()
            temp_bytes = _native.check_size(lib.vgr_lidar_ray_order_temp_bytes(rays), "ray order")
            # Buffers are reused while the ray count and device stay the same.
            if self._order is None or self._order.shape[0] != rays or self._order.device != directions.device:
                self._order = torch.empty((rays,), dtype=torch.int32, device=directions.device)
                self._temp = torch.empty((temp_bytes,), dtype=torch.uint8, device=directions.device)
            stream = torch.cuda.current_stream(directions.device).cuda_stream
            _native.check(
                lib.vgr_lidar_ray_order(directions.data_ptr(), rays, self._order.data_ptr(),
                                        self._temp.data_ptr(), temp_bytes, stream),
                "ray order",
            )
            self._key = key
        return self._order


def native_scene(scene: GaussianLidarScene) -> VgrLidarScene:
    return VgrLidarScene(
        means=scene.means.data_ptr(),
        scales=scene.scales.data_ptr(),
        rotations=scene.rotations.data_ptr(),
        opacities=scene.opacities.data_ptr(),
        semantic_ids=scene.semantic_ids.data_ptr(),
        reflectivity=None if scene.reflectivity is None else scene.reflectivity.data_ptr(),
        surface_confidence=None if scene.surface_confidence is None else scene.surface_confidence.data_ptr(),
        count=scene.count,
    )


class CudaLidarBackend:
    def __init__(
        self,
        *,
        max_scenes: int = 64,
        packet_size: int = 8,
        near_plane_m: float = 0.05,
        far_plane_m: float = 200.0,
        support_sigma: float = 3.0,
        detection_threshold: float = 0.01,
        planarity_ratio_max: float = 0.35,
        min_incidence_cos: float = 0.05,
        cluster_abs_m: float = 0.02,
        cluster_relative: float = 0.001,
        fallback_reflectivity: float = 0.5,
        direction_norm_tolerance: float = 1.0e-4,
        semantic_slots: int = 16,
        native_module: Any | None = None,
        allow_cpu_for_tests: bool = False,
    ) -> None:
        if max_scenes <= 0:
            raise ValueError("max_scenes must be positive.")
        if packet_size not in (8, 16):
            raise ValueError("packet_size must be 8 or 16.")
        if near_plane_m <= 0 or far_plane_m <= near_plane_m:
            raise ValueError("Expected 0 < near_plane_m < far_plane_m.")
        if support_sigma <= 0:
            raise ValueError("support_sigma must be positive.")
        if not 0 < detection_threshold <= 1:
            raise ValueError("detection_threshold must be in (0, 1].")
        if not 0 < planarity_ratio_max <= 1:
            raise ValueError("planarity_ratio_max must be in (0, 1].")
        if not 0 < min_incidence_cos <= 1:
            raise ValueError("min_incidence_cos must be in (0, 1].")
        if cluster_abs_m < 0 or cluster_relative < 0:
            raise ValueError("cluster thresholds must be non-negative.")
        if not 0 <= fallback_reflectivity <= 1:
            raise ValueError("fallback_reflectivity must be in [0, 1].")
        if not 0 < direction_norm_tolerance < 1:
            raise ValueError("direction_norm_tolerance must be in (0, 1).")
        if semantic_slots <= 0 or semantic_slots > 32:
            raise ValueError("semantic_slots must be in [1, 32].")
        self.max_scenes = max_scenes
        self.packet_size = packet_size
        self.near_plane_m = near_plane_m
        self.far_plane_m = far_plane_m
        self.support_sigma = support_sigma
        self.detection_threshold = detection_threshold
        self.planarity_ratio_max = planarity_ratio_max
        self.min_incidence_cos = min_incidence_cos
        self.cluster_abs_m = cluster_abs_m
        self.cluster_relative = cluster_relative
        self.fallback_reflectivity = fallback_reflectivity
        self.direction_norm_tolerance = direction_norm_tolerance
        self.semantic_slots = semantic_slots
        self._native = native_module
        self.allow_cpu_for_tests = allow_cpu_for_tests
        self.device: torch.device | None = None
        self.stage: Any | None = None
        self.workspace: dict[str, torch.Tensor] = {}
        self._scenes: OrderedDict[int, _SceneAcceleration] = OrderedDict()
        self._ray_order = RayOrder()

    # ------------------------------------------------------------ lifecycle
    def initialize(self, stage: Any, device: torch.device) -> None:
        device = torch.device(device)
        if device.type != "cuda" and not self.allow_cpu_for_tests:
            raise ValueError(f"CudaLidarBackend requires CUDA; got {device}.")
        self.stage = stage
        self.device = device
        if device.type == "cuda":
            _native.load_library()

    def allocate_workspace(self, *, max_sensors: int, max_rays: int, device: torch.device) -> dict[str, torch.Tensor]:
        self._require_initialized()
        identity = torch.eye(4, device=device, dtype=torch.float32)
        rows = (LIDAR_DESCRIPTOR_BYTES + 7) // 8
        self.workspace = {
            "scene_descriptors": torch.zeros((self.max_scenes, rows), device=device, dtype=torch.int64),
            "counters": torch.zeros((len(LIDAR_COUNTER_NAMES),), device=device, dtype=torch.int64),
            "identity_scene_to_world": identity.repeat(max_sensors, 1, 1).contiguous(),
            "all_active_sensor_ids": torch.arange(max_sensors, device=device, dtype=torch.int64),
        }
        return self.workspace

    def register_scene(self, scene_id: int, scene: GaussianLidarScene) -> None:
        self._require_workspace()
        if scene_id in self._scenes:
            raise ValueError(f"LiDAR scene {scene_id} is already registered.")
        if len(self._scenes) >= self.max_scenes:
            raise ValueError(f"LiDAR scene count exceeds max_scenes={self.max_scenes}.")
        lib = _native.load_library()
        nbytes = _native.check_size(lib.vgr_lidar_sort_temp_bytes(scene.count, self.packet_size), "lidar accel")
        accel = torch.empty((nbytes,), dtype=torch.uint8, device=self.device)
        acceleration = _SceneAcceleration(scene=scene, accel=accel)
        self._scenes[scene_id] = acceleration
        self._build_and_pack(len(self._scenes) - 1, scene_id, acceleration)

    def revise_scene(self, scene_id: int, scene: GaussianLidarScene) -> None:
        self._require_workspace()
        if scene_id not in self._scenes:
            raise ValueError(f"Unregistered LiDAR scene ID: {scene_id}.")
        acceleration = self._scenes[scene_id]
        if scene.count != acceleration.scene.count:
            raise ValueError("A scene revision must retain the registered Gaussian count.")
        acceleration.scene = scene
        self._build_and_pack(tuple(self._scenes).index(scene_id), scene_id, acceleration)

    def rebuild_scene(self, scene_id: int) -> None:
        """Rebuild one scene's acceleration in place (steady-state frame rebuilds;
        no allocation, no host synchronisation)."""
        acceleration = self._scenes[scene_id]
        self._build(acceleration)

    def render_lidar(self, request: LidarRenderRequest) -> None:
        self._require_workspace()
        if not self._scenes:
            raise RuntimeError("At least one Gaussian LiDAR scene must be registered.")
        lib = _native.load_library()
        inputs = VgrLidarInputs(
            ray_directions=request.ray_directions.data_ptr(),
            rays=request.ray_directions.shape[0],
            time_offsets=request.time_offsets_ns.data_ptr(),
            time_offsets_are_int64=int(request.time_offsets_ns.dtype == torch.int64),
            sensor_to_world=request.sensor_to_world.data_ptr(),
            scene_to_world=request.scene_to_world.data_ptr(),
            scene_ids=request.scene_ids.data_ptr(),
            batch=request.sensor_to_world.shape[0],
            active_sensor_ids=None if request.active_sensor_ids is None else request.active_sensor_ids.data_ptr(),
            active_count=0 if request.active_sensor_ids is None else request.active_sensor_ids.numel(),
            ray_order=self._ray_order(request.ray_directions).data_ptr(),
        )
        out = request.outputs
        outputs = VgrLidarOutputs(
            range_m=out["range_m"].data_ptr(),
            position_world_m=out["position_world_m"].data_ptr(),
            intensity=out["intensity"].data_ptr(),
            semantic_id=out["semantic_id"].data_ptr(),
            valid=out["valid"].data_ptr(),
            time_offset_ns=out["time_offset_ns"].data_ptr(),
            return_count=out["return_count"].data_ptr(),
        )
        with torch.cuda.device(self.device):
            stream = torch.cuda.current_stream(self.device).cuda_stream
            with torch.cuda.nvtx.range("GaussianLidarService.render_lidar"):
                _native.check(
                    lib.vgr_render_lidar(
                        self.workspace["scene_descriptors"].data_ptr(),
                        len(self._scenes),
                        inputs,
                        outputs,
                        self.workspace["counters"].data_ptr(),
                        self._options(request.returns),
                        stream,
                    ),
                    "render_lidar",
                )

    def synchronize(self) -> None:
        self._require_initialized()
        if self.device is not None and self.device.type == "cuda":
            torch.cuda.synchronize(self.device)

    def read_counters(self, *, synchronize: bool = True) -> dict[str, int]:
        if synchronize:
            self.synchronize()
        values = self.workspace["counters"].detach().cpu().tolist()
        return dict(zip(LIDAR_COUNTER_NAMES, (int(v) for v in values)))

    def check_errors(self, *, synchronize: bool = True) -> dict[str, int]:
        counters = self.read_counters(synchronize=synchronize)
        errors = {
            name: counters[name]
            for name in (
                "stack_overflow",
                "semantic_overflow",
                "invalid_directions",
                "invalid_scene_ids",
                "invalid_active_sensor_ids",
            )
            if counters[name]
        }
        if errors:
            raise LidarTraversalError(f"Gaussian LiDAR device errors: {errors}.")
        return counters

    def surfel_count(self, scene_id: int) -> int:
        """Planar surfels of the scene's current build (the device-computed
        count in the acceleration header; synchronises)."""
        accel = self._scenes[scene_id].accel
        return int(accel[:4].view(torch.int32).item())

    @property
    def bvh_bytes(self) -> int:
        return sum(acc.bvh_bytes for acc in self._scenes.values())

    @property
    def scene_attribute_bytes(self) -> int:
        total = 0
        for acc in self._scenes.values():
            s = acc.scene
            for t in (s.means, s.scales, s.rotations, s.opacities, s.semantic_ids, s.reflectivity, s.surface_confidence):
                if t is not None:
                    total += t.numel() * t.element_size()
        return total

    @property
    def workspace_bytes(self) -> int:
        return sum(t.numel() * t.element_size() for t in self.workspace.values())

    def shutdown(self) -> None:
        if self.device is not None and self.device.type == "cuda":
            self.synchronize()
        self.workspace = {}
        self._scenes.clear()
        self.stage = None
        self.device = None

    # --------------------------------------------------------------- helpers
    def _options(self, returns: int) -> VgrLidarOptions:
        return VgrLidarOptions(
            returns=returns,
            semantic_slots=self.semantic_slots,
            near_plane_m=self.near_plane_m,
            far_plane_m=self.far_plane_m,
            support_sigma=self.support_sigma,
            detection_threshold=self.detection_threshold,
            planarity_ratio_max=self.planarity_ratio_max,
            min_incidence_cos=self.min_incidence_cos,
            cluster_abs_m=self.cluster_abs_m,
            cluster_relative=self.cluster_relative,
            fallback_reflectivity=self.fallback_reflectivity,
            direction_norm_tolerance=self.direction_norm_tolerance,
        )

    def _build(self, acceleration: _SceneAcceleration) -> None:
        lib = _native.load_library()
        with torch.cuda.device(self.device):
            stream = torch.cuda.current_stream(self.device).cuda_stream
            _native.check(
                lib.vgr_lidar_build_scene_lbvh(
                    native_scene(acceleration.scene),
                    self.packet_size,
                    self.support_sigma,
                    self.planarity_ratio_max,
                    acceleration.accel.data_ptr(),
                    acceleration.accel.numel(),
                    stream,
                ),
                "build_scene_lbvh",
            )

    def _build_and_pack(self, slot: int, scene_id: int, acceleration: _SceneAcceleration) -> None:
        self._build(acceleration)
        lib = _native.load_library()
        with torch.cuda.device(self.device):
            stream = torch.cuda.current_stream(self.device).cuda_stream
            _native.check(
                lib.vgr_lidar_pack_scene_descriptor(
                    self.workspace["scene_descriptors"].data_ptr(),
                    self.max_scenes,
                    slot,
                    scene_id,
                    acceleration.accel.data_ptr(),
                    acceleration.scene.count,
                    self.packet_size,
                    stream,
                ),
                "pack_scene_descriptor",
            )

    def _require_initialized(self) -> None:
        if self.device is None:
            raise RuntimeError("CudaLidarBackend.initialize(stage, device) must be called first.")

    def _require_workspace(self) -> None:
        self._require_initialized()
        if not self.workspace:
            raise RuntimeError("allocate_workspace() must be called first.")
