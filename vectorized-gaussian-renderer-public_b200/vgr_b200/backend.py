"""Backend protocol of the renderer service (the plugin seam).

Mirrors src/isaacsim_gaussian_renderer/backend.py:10-67: the service passes
validated tensors in a RenderRequest and the backend renders into the
request's output tensors.
"""

from __future__ import annotations

from dataclasses import dataclass, field
from typing import Any, Protocol

import torch


@dataclass(frozen=True)
class RenderStats:
    rendered_views: int
    visible_gaussians: int | None = None
    tile_intersections: int | None = None


@dataclass(frozen=True)
class RenderRequest:
    camera_transforms: torch.Tensor
    intrinsics: torch.Tensor
    scene_ids: torch.Tensor
    scene_offsets: torch.Tensor
    outputs: dict[str, torch.Tensor]
    active_camera_ids: torch.Tensor | None = None
    workspace: dict[str, torch.Tensor] = field(default_factory=dict)


class GaussianRendererBackend(Protocol):
    def initialize(self, stage: Any, device: torch.device) -> None: ...

    def register_scene(self, scene_id: int, scene: Any, offset: int) -> None: ...

    def allocate_workspace(
        self,
        *,
        max_views: int,
        height: int,
        width: int,
        device: torch.device,
        dtype: torch.dtype,
    ) -> dict[str, torch.Tensor]: ...

    def update_scene_transforms(self, scene_ids: torch.Tensor, transforms: torch.Tensor) -> None: ...

    def render(self, request: RenderRequest) -> RenderStats: ...

    def synchronize(self) -> None: ...

    def shutdown(self) -> None: ...
