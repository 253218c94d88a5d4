"""Caller-owned Gaussian scenes and the packed-offset registry.

Public surface of src/isaacsim_gaussian_renderer/scene.py:12-127
(``GaussianScene`` with ``count``/``validate``, ``SceneRegistry`` with
``scene_ids``, ``total_gaussians``, ``register``, ``require_scene_ids`` and
``offsets_tensor``, the same ValueError texts).  Layout: float32 means
[G,3], activated scales [G,3], WXYZ rotations [G,4], activated opacities
[G], features [G,F] (linear RGB in the first three channels, or the
[(d+1)^2, 3] spherical-harmonics coefficients of the SH colour mode) and
int64 semantic ids [G].

The registry is one ``SceneTable`` of per-scene Gaussian counts; the packed
offsets are their running sum, rebuilt as one int64 tensor per device the
first time a device asks after a registration.
"""

from __future__ import annotations

from dataclasses import dataclass
from itertools import accumulate

import torch

from ._service_core import SceneTable, TensorField, check_fields

SCENE_FIELDS: tuple[TensorField, ...] = (
    TensorField("means", (3,), torch.float32, free_leading=True),
    TensorField("scales", (3,), torch.float32),
    TensorField("rotations", (4,), torch.float32),
    TensorField("opacities", (), torch.float32),
    TensorField("features", (None,), torch.float32),
    TensorField("semantic_ids", (), torch.int64),
)


@dataclass(frozen=True)
class GaussianScene:
    means: torch.Tensor
    scales: torch.Tensor
    rotations: torch.Tensor
    opacities: torch.Tensor
    features: torch.Tensor
    semantic_ids: torch.Tensor

    @property
    def count(self) -> int:
        return int(self.means.shape[0])

    def validate(self, *, device: torch.device, require_cuda: bool) -> "GaussianScene":
        check_fields(self, SCENE_FIELDS, self.count, device=device, require_cuda=require_cuda)
        return self


class SceneRegistry:
    """Scene id -> scene, and the packed offsets of the concatenated scenes
    in registration order (the order the backend packs them)."""

    def __init__(self) -> None:
        self._table: SceneTable[GaussianScene] = SceneTable("scene")
        self._per_device: dict[torch.device, torch.Tensor] = {}

    @property
    def scene_ids(self) -> tuple[int, ...]:
        return self._table.ids

    @property
    def total_gaussians(self) -> int:
        return sum(scene.count for scene in self._table.values())

    def offsets(self) -> list[int]:
        """[S+1] running sum of the registered scenes' Gaussian counts."""
        return list(accumulate((scene.count for scene in self._table.values()), initial=0))

    def register(self, scene_id: int, scene: GaussianScene) -> int:
        """Add a scene after the ones already packed; returns its offset."""
        start = self.total_gaussians
        self._table.insert(scene_id, scene)
        self._per_device = {}
        return start

    def require_scene_ids(self, scene_ids: torch.Tensor) -> None:
        self._table.check_host_ids(scene_ids)

    def offsets_tensor(self, *, device: torch.device, require_cuda: bool) -> torch.Tensor:
        if device not in self._per_device:
            self._per_device[device] = torch.tensor(self.offsets(), dtype=torch.int64, device=device)
        offsets = self._per_device[device]
        if require_cuda and offsets.device.type != "cuda":
            raise ValueError("scene_offsets must be CUDA-resident.")
        return offsets
