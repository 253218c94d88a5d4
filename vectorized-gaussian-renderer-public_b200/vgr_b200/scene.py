"""Caller-owned Gaussian scenes and the packed-offset registry.

Same canonical layout and validation as the reference
(src/isaacsim_gaussian_renderer/scene.py:12-127): float32 means [G,3],
activated scales [G,3], WXYZ rotations [G,4], activated opacities [G],
features [G,F] whose first three channels are linear RGB (or, for the
spherical-harmonics colour mode, [(d+1)^2, 3] coefficients per Gaussian),
and int64 semantic ids [G].
"""

from __future__ import annotations

from dataclasses import dataclass

import torch

from .contracts import ensure_tensor


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
        count = self.count
        specs = (
            ("means", self.means, (None, 3), torch.float32),
            ("scales", self.scales, (count, 3), torch.float32),
            ("rotations", self.rotations, (count, 4), torch.float32),
            ("opacities", self.opacities, (count,), torch.float32),
            ("features", self.features, (count, None), torch.float32),
            ("semantic_ids", self.semantic_ids, (count,), torch.int64),
        )
        for name, tensor, shape, dtype in specs:
            ensure_tensor(
                tensor,
                name=name,
                shape=shape,
                dtype=dtype,
                device=device,
                require_cuda=require_cuda,
            )
        return self


class SceneRegistry:
    """Scene id -> scene, with the packed offsets of the concatenated scenes."""

    def __init__(self) -> None:
        self._scenes: dict[int, GaussianScene] = {}
        self._offsets: list[int] = [0]
        self._offset_tensors: dict[torch.device, torch.Tensor] = {}

    @property
    def scene_ids(self) -> tuple[int, ...]:
        return tuple(self._scenes)

    @property
    def total_gaussians(self) -> int:
        return self._offsets[-1]

    def register(self, scene_id: int, scene: GaussianScene) -> int:
        if scene_id in self._scenes:
            raise ValueError(f"Scene {scene_id} is already registered.")
        offset = self._offsets[-1]
        self._scenes[scene_id] = scene
        self._offsets.append(offset + scene.count)
        self._offset_tensors.clear()
        return offset

    def require_scene_ids(self, scene_ids: torch.Tensor) -> None:
        if scene_ids.device.type != "cpu":
            raise ValueError("Host scene-ID validation accepts CPU tensors only.")
        missing = sorted({int(v) for v in scene_ids.tolist()} - set(self._scenes))
        if missing:
            raise ValueError(f"Unregistered scene ID(s): {missing}.")

    def offsets_tensor(self, *, device: torch.device, require_cuda: bool) -> torch.Tensor:
        tensor = self._offset_tensors.get(device)
        if tensor is None:
            tensor = torch.tensor(self._offsets, dtype=torch.int64, device=device)
            self._offset_tensors[device] = tensor
        if require_cuda and tensor.device.type != "cuda":
            raise ValueError("scene_offsets must be CUDA-resident.")
        return tensor
