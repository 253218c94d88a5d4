"""Public, explicitly constructed Gaussian LiDAR service.

Call surface of src/isaacsim_gaussian_renderer/lidar_service.py:20-220:
initialize, load_scene (with optional reflectivity/surface confidence and a
revision), revise_scene, render_lidar (shared sensor-local rays, per-sensor
scene ids and transforms, optional strictly increasing active sensors,
caller- or service-owned outputs, K in {1, 2}), synchronize, shutdown; same
arguments and error texts.  Every call rewrites every output; there is no
cadence and no private stream.

Structure as the camera service: a ``ServiceLifecycle`` (device, guard), a
``LidarSceneRegistry`` (scenes and revisions) and an ``OutputSetPool`` of
service-owned outputs keyed by (sensors, rays, returns); ``render_lidar``
validates and forwards one ``LidarRenderRequest``.
"""

from __future__ import annotations

from typing import Any

import torch

from ._service_core import OutputSetPool, ServiceLifecycle
from .lidar_backend import GaussianLidarBackend, LidarRenderRequest
from .lidar_contracts import (
    LIDAR_OUTPUT_SPECS,
    lidar_output_shape,
    validate_active_sensor_ids,
    validate_lidar_outputs,
    validate_lidar_request,
    validate_scene_transforms,
)
from .lidar_scene import GaussianLidarScene, LidarSceneRegistry

_RETURNS_MESSAGE = "returns must be exactly 1 or 2."


class GaussianLidarService:
    mode = "gaussian_surface"

    def __init__(
        self,
        backend: GaussianLidarBackend,
        *,
        max_sensors: int,
        max_rays: int,
        returns: int = 1,
        allow_cpu_for_tests: bool = False,
    ) -> None:
        if min(max_sensors, max_rays) <= 0:
            raise ValueError("max_sensors and max_rays must be positive.")
        if returns not in (1, 2):
            raise ValueError(_RETURNS_MESSAGE)
        self.backend = backend
        self.max_sensors = max_sensors
        self.max_rays = max_rays
        self.returns = returns
        self.allow_cpu_for_tests = allow_cpu_for_tests
        self.stage: Any | None = None
        self.registry = LidarSceneRegistry()
        self.workspace: dict[str, torch.Tensor] = {}
        self._life = ServiceLifecycle("GaussianLidarService", allow_cpu_for_tests)
        self._outputs = OutputSetPool(self._new_output_set)

    @property
    def device(self) -> torch.device | None:
        return self._life.device

    # ------------------------------------------------------------ lifecycle
    def initialize(self, stage: Any, device: torch.device | str) -> None:
        resolved = self._life.start(device)
        self.stage = stage
        self.backend.initialize(stage, resolved)
        self.workspace = self.backend.allocate_workspace(
            max_sensors=self.max_sensors, max_rays=self.max_rays, device=resolved
        )
        self._life.ready = True

    def synchronize(self) -> None:
        self._life.check()
        self.backend.synchronize()

    def shutdown(self) -> None:
        if self._life.ready:
            self.backend.shutdown()
        self._life.ready = False
        self.workspace = {}
        self._outputs.clear()

    # ---------------------------------------------------------------- scenes
    def load_scene(
        self,
        scene_id: int,
        *,
        means: torch.Tensor,
        scales: torch.Tensor,
        rotations: torch.Tensor,
        opacities: torch.Tensor,
        semantic_ids: torch.Tensor,
        reflectivity: torch.Tensor | None = None,
        surface_confidence: torch.Tensor | None = None,
        revision: int = 0,
    ) -> None:
        device = self._life.check()
        scene = GaussianLidarScene(means, scales, rotations, opacities, semantic_ids, reflectivity,
                                   surface_confidence, revision)
        scene.validate(device=device, require_cuda=self._life.require_cuda)
        self.registry.register(scene_id, scene)
        self.backend.register_scene(scene_id, scene)

    def revise_scene(self, scene_id: int, *, revision: int) -> None:
        """Rebuild the scene's acceleration after same-storage geometry edits."""
        device = self._life.check()

        def validated(candidate: GaussianLidarScene) -> GaussianLidarScene:
            return candidate.validate(device=device, require_cuda=self._life.require_cuda)

        self.backend.revise_scene(scene_id, self.registry.revise(scene_id, revision, validate=validated))

    # --------------------------------------------------------------- render
    def render_lidar(
        self,
        ray_directions: torch.Tensor,
        time_offsets_ns: torch.Tensor,
        sensor_to_world: torch.Tensor,
        scene_ids: torch.Tensor,
        *,
        scene_to_world: torch.Tensor | None = None,
        active_sensor_ids: torch.Tensor | None = None,
        outputs: dict[str, torch.Tensor] | None = None,
        returns: int | None = None,
    ) -> dict[str, torch.Tensor]:
        device = self._life.check()
        cuda = self._life.require_cuda
        k = returns if returns is not None else self.returns
        if k not in (1, 2):
            raise ValueError(_RETURNS_MESSAGE)
        batch, rays = validate_lidar_request(ray_directions, time_offsets_ns, sensor_to_world, scene_ids,
                                             device=device, require_cuda=cuda)
        if batch > self.max_sensors or rays > self.max_rays:
            raise ValueError(
                f"Request B={batch}, R={rays} exceeds configured B={self.max_sensors}, R={self.max_rays}."
            )
        active_sensor_ids = validate_active_sensor_ids(active_sensor_ids, batch=batch, device=device,
                                                       require_cuda=cuda)
        if not cuda:
            self.registry.require_scene_ids(scene_ids)
        if scene_to_world is not None:
            validate_scene_transforms(scene_to_world, batch=batch, device=device, require_cuda=cuda)
        else:
            scene_to_world = self.workspace["identity_scene_to_world"][:batch]
        target = self._outputs.get((batch, rays, k)) if outputs is None else outputs
        validate_lidar_outputs(target, batch=batch, rays=rays, returns=k, device=device, require_cuda=cuda)
        self.backend.render_lidar(
            LidarRenderRequest(
                ray_directions=ray_directions,
                time_offsets_ns=time_offsets_ns,
                sensor_to_world=sensor_to_world,
                scene_to_world=scene_to_world,
                scene_ids=scene_ids,
                outputs=target,
                returns=k,
                active_sensor_ids=active_sensor_ids,
            )
        )
        return target

    def _new_output_set(self, key: tuple[int, int, int]) -> dict[str, torch.Tensor]:
        batch, rays, k = key
        return {
            name: torch.empty(lidar_output_shape(name, batch, rays, k), dtype=dtype, device=self.device)
            for name, dtype in LIDAR_OUTPUT_SPECS.items()
        }
