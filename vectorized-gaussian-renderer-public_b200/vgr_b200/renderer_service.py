"""Public camera renderer service.

Call surface of the reference ``RendererService``
(src/isaacsim_gaussian_renderer/renderer_service.py:14-237): initialize,
load_scene, update_scene_transforms, prepare_outputs, render (with optional
caller-owned outputs and device-resident active camera ids), synchronize,
shutdown, a render cadence (``render_every_n``) and service-owned outputs
that start at the inactive contract (zeros, semantic -1); same arguments,
ValueError/RuntimeError texts and workspace identity.

Structure: a ``ServiceLifecycle`` owns the device and the
initialise-before-use guard, a ``SceneRegistry`` the packed offsets, an
``OutputSetPool`` the service-owned outputs by batch size, and
``RenderCadence`` decides which requests reach the backend.  ``render``
validates the request (shapes, dtypes, residency; ids only for CPU tensors,
never by reading device memory back), then either forwards one
``RenderRequest`` or returns the previous outputs.
"""

from __future__ import annotations

from collections.abc import Iterable
from typing import Any

import torch

from ._service_core import OutputSetPool, ServiceLifecycle
from .backend import GaussianRendererBackend, RenderRequest
from .contracts import (
    OUTPUT_SPECS,
    ensure_tensor,
    validate_active_camera_ids,
    validate_camera_batch,
    validate_outputs,
)
from .scene import GaussianScene, SceneRegistry


class RenderCadence:
    """Every n-th request renders, the first one included; the others return
    the last rendered outputs."""

    def __init__(self, every_n: int) -> None:
        if every_n <= 0:
            raise ValueError("render_every_n must be positive.")
        self.every_n = every_n
        self.requests = 0
        self.last: dict[str, torch.Tensor] | None = None

    def admit(self) -> bool:
        self.requests += 1
        return (self.requests - 1) % self.every_n == 0

    def replay(self) -> dict[str, torch.Tensor]:
        if self.last is None:
            raise RuntimeError("Render cadence skipped before any output exists.")
        return self.last


class RendererService:
    def __init__(
        self,
        backend: GaussianRendererBackend,
        *,
        height: int,
        width: int,
        outputs: Iterable[str] = ("rgb", "depth", "alpha", "semantic_id"),
        max_views: int | None = None,
        render_every_n: int = 1,
        allow_cpu_for_tests: bool = False,
    ) -> None:
        if min(height, width) <= 0:
            raise ValueError("height and width must be positive.")
        self._cadence = RenderCadence(render_every_n)
        self.output_names = tuple(outputs)
        unsupported = [name for name in sorted(set(self.output_names)) if name not in OUTPUT_SPECS]
        if unsupported:
            raise ValueError(f"Unsupported output name(s): {', '.join(unsupported)}.")
        self.backend = backend
        self.height = height
        self.width = width
        self.max_views = max_views
        self.render_every_n = render_every_n
        self.allow_cpu_for_tests = allow_cpu_for_tests
        self.stage: Any | None = None
        self.registry = SceneRegistry()
        self.workspace: dict[str, torch.Tensor] = {}
        self._life = ServiceLifecycle("RendererService", allow_cpu_for_tests)
        self._outputs = OutputSetPool(self._new_output_set,
                                      still_valid=lambda found: tuple(found) == self.output_names)

    @property
    def device(self) -> torch.device | None:
        return self._life.device

    # ------------------------------------------------------------ lifecycle
    def initialize(self, stage: Any, device: torch.device | str) -> None:
        resolved = self._life.start(device)
        self.stage = stage
        self.backend.initialize(stage, resolved)
        if self.max_views is not None:
            self.workspace = self.backend.allocate_workspace(
                max_views=self.max_views, height=self.height, width=self.width, device=resolved,
                dtype=torch.float32,
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
        self._cadence.last = None

    # ---------------------------------------------------------------- scenes
    def load_scene(
        self,
        scene_id: int,
        *,
        means: torch.Tensor,
        scales: torch.Tensor,
        rotations: torch.Tensor,
        opacities: torch.Tensor,
        features: torch.Tensor,
        semantic_ids: torch.Tensor,
    ) -> None:
        device = self._life.check()
        scene = GaussianScene(means, scales, rotations, opacities, features, semantic_ids)
        scene.validate(device=device, require_cuda=self._life.require_cuda)
        self.backend.register_scene(scene_id, scene, self.registry.register(scene_id, scene))
        # The packed offsets are materialised here so render() never allocates them.
        self.registry.offsets_tensor(device=device, require_cuda=self._life.require_cuda)

    def update_scene_transforms(self, scene_ids: torch.Tensor, transforms: torch.Tensor) -> None:
        device = self._life.check()
        cuda = self._life.require_cuda
        ensure_tensor(transforms, name="transforms", shape=(None, 4, 4), dtype=torch.float32, device=device,
                      require_cuda=cuda)
        count = transforms.shape[0]
        if tuple(scene_ids.shape) != (count,):
            raise ValueError("scene_ids must have one entry per transform.")
        ensure_tensor(scene_ids, name="scene_ids", shape=(count,), dtype=torch.int64, device=device,
                      require_cuda=cuda)
        if not cuda:
            self.registry.require_scene_ids(scene_ids)
        self.backend.update_scene_transforms(scene_ids, transforms)

    # --------------------------------------------------------------- render
    def prepare_outputs(self, batch: int) -> dict[str, torch.Tensor]:
        """Allocate and retain one logical output set before steady state."""
        self._life.check()
        if batch <= 0:
            raise ValueError("batch must be positive.")
        self._check_batch(batch)
        return self._outputs.get(batch)

    def render(
        self,
        camera_transforms: torch.Tensor,
        intrinsics: torch.Tensor,
        scene_ids: torch.Tensor,
        outputs: dict[str, torch.Tensor] | None = None,
        active_camera_ids: torch.Tensor | None = None,
    ) -> dict[str, torch.Tensor]:
        device = self._life.check()
        cuda = self._life.require_cuda
        batch = validate_camera_batch(camera_transforms, intrinsics, scene_ids, device=device, require_cuda=cuda)
        self._check_batch(batch)
        active_camera_ids = validate_active_camera_ids(active_camera_ids, batch=batch, device=device,
                                                       require_cuda=cuda)
        if not cuda:
            self.registry.require_scene_ids(scene_ids)
        target = self._outputs.get(batch) if outputs is None else outputs
        validate_outputs(target, batch=batch, height=self.height, width=self.width, device=device,
                         require_cuda=cuda)
        if not self._cadence.admit():
            return self._cadence.replay()
        self.backend.render(
            RenderRequest(
                camera_transforms=camera_transforms,
                intrinsics=intrinsics,
                scene_ids=scene_ids,
                scene_offsets=self.registry.offsets_tensor(device=device, require_cuda=cuda),
                outputs=target,
                active_camera_ids=active_camera_ids,
                workspace=self.workspace,
            )
        )
        self._cadence.last = target
        return target

    # -------------------------------------------------------------- helpers
    def _check_batch(self, batch: int) -> None:
        if self.max_views is not None and batch > self.max_views:
            raise ValueError(f"Batch has {batch} cameras but service max_views is {self.max_views}.")

    def _new_output_set(self, batch: int) -> dict[str, torch.Tensor]:
        """One output set at the inactive contract: zeros, semantic -1."""
        owned: dict[str, torch.Tensor] = {}
        for name in self.output_names:
            channels, dtype = OUTPUT_SPECS[name]
            fill = -1 if name == "semantic_id" else 0
            owned[name] = torch.full((batch, self.height, self.width, channels), fill, dtype=dtype,
                                     device=self.device)
        return owned
