"""Gaussian LiDAR scenes and explicit revision tracking.

Public surface of src/isaacsim_gaussian_renderer/lidar_scene.py:13-152
(``GaussianLidarScene`` with ``count``/``validate``, ``LidarSceneRegistry``
with ``scene_ids``, ``register``, ``scene``, ``revise`` and
``require_scene_ids``, the same ValueError texts): caller-owned tensors, WXYZ
rotations, activated scales, opacity, reflectivity and confidence in their
ranges, non-negative semantic ids (-1 is the no-hit value) and explicit
monotone revisions that trigger an acceleration rebuild.

Validation is two tables: the tensor fields (shape/dtype/device, checked by
``check_fields``) and the value rules, each a predicate over the scene with
the message it raises.  Registration is a cold path, so the value rules may
synchronise.
"""

from __future__ import annotations

import dataclasses
from collections.abc import Callable
from dataclasses import dataclass

import torch

from ._service_core import SceneTable, TensorField, check_fields

LIDAR_SCENE_FIELDS: tuple[TensorField, ...] = (
    TensorField("means", (3,), torch.float32, free_leading=True),
    TensorField("scales", (3,), torch.float32),
    TensorField("rotations", (4,), torch.float32),
    TensorField("opacities", (), torch.float32),
    TensorField("semantic_ids", (), torch.int64),
    TensorField("reflectivity", (), torch.float32, optional=True),
    TensorField("surface_confidence", (), torch.float32, optional=True),
)


def _unit_interval(tensor: torch.Tensor | None) -> bool:
    return tensor is None or bool(torch.isfinite(tensor).all() and tensor.min() >= 0 and tensor.max() <= 1)


def _unit_quaternions(rotations: torch.Tensor) -> bool:
    norms = torch.linalg.vector_norm(rotations, dim=1)
    return bool(((norms - 1.0).abs() <= 1.0e-4).all())


# (predicate that must hold, message when it does not), in checking order.
LIDAR_VALUE_RULES: tuple[tuple[Callable[["GaussianLidarScene"], bool], str], ...] = (
    (lambda s: bool(torch.isfinite(s.means).all()), "means must be finite."),
    (lambda s: bool(torch.isfinite(s.scales).all() and s.scales.min() > 0), "scales must be finite and positive."),
    (lambda s: bool(s.semantic_ids.min() >= 0),
     "semantic_ids must be non-negative; -1 is reserved for no-hit outputs."),
    (lambda s: _unit_quaternions(s.rotations), "rotations must be normalized WXYZ quaternions."),
    (lambda s: _unit_interval(s.opacities), "opacities must be finite and in [0, 1]."),
    (lambda s: _unit_interval(s.reflectivity), "reflectivity must be finite and in [0, 1]."),
    (lambda s: _unit_interval(s.surface_confidence), "surface_confidence must be finite and in [0, 1]."),
)


@dataclass(frozen=True)
class GaussianLidarScene:
    means: torch.Tensor
    scales: torch.Tensor
    rotations: torch.Tensor
    opacities: torch.Tensor
    semantic_ids: torch.Tensor
    reflectivity: torch.Tensor | None = None
    surface_confidence: torch.Tensor | None = None
    revision: int = 0

    @property
    def count(self) -> int:
        return int(self.means.shape[0])

    def validate(self, *, device: torch.device, require_cuda: bool) -> "GaussianLidarScene":
        if self.revision < 0:
            raise ValueError("scene revision must be non-negative.")
        if self.count <= 0:
            raise ValueError("A Gaussian LiDAR scene must contain at least one Gaussian.")
        check_fields(self, LIDAR_SCENE_FIELDS, self.count, device=device, require_cuda=require_cuda)
        for holds, message in LIDAR_VALUE_RULES:
            if not holds(self):
                raise ValueError(message)
        return self


class LidarSceneRegistry:
    """One caller-owned scene and its current revision per scene id."""

    def __init__(self) -> None:
        self._table: SceneTable[GaussianLidarScene] = SceneTable("LiDAR scene")

    @property
    def scene_ids(self) -> tuple[int, ...]:
        return self._table.ids

    def register(self, scene_id: int, scene: GaussianLidarScene) -> None:
        self._table.insert(scene_id, scene)

    def scene(self, scene_id: int) -> GaussianLidarScene:
        return self._table.lookup(scene_id)

    def revise(
        self,
        scene_id: int,
        revision: int,
        *,
        validate: Callable[[GaussianLidarScene], GaussianLidarScene] | None = None,
    ) -> GaussianLidarScene:
        """The same tensors under a strictly larger revision number
        (validated by ``validate`` before it replaces the current entry)."""
        current = self._table.lookup(scene_id)
        if not revision > current.revision:
            raise ValueError(
                f"LiDAR scene {scene_id} revision must increase from {current.revision}; got {revision}."
            )
        revised = dataclasses.replace(current, revision=revision)
        revised = validate(revised) if validate is not None else revised
        self._table.replace(scene_id, revised)
        return revised

    def require_scene_ids(self, scene_ids: torch.Tensor) -> None:
        self._table.check_host_ids(scene_ids)
