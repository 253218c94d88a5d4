"""Pieces shared by the camera and LiDAR services.

The services keep the reference's public call surface and error messages
(src/isaacsim_gaussian_renderer/renderer_service.py, lidar_service.py,
scene.py, lidar_scene.py); the structure underneath is this module's:

* ``TensorField`` tables describe a scene's tensors once and
  ``check_fields`` validates any dataclass against its table;
* ``ServiceLifecycle`` resolves the device and guards calls made before
  ``initialize``;
* ``SceneTable`` is the insertion-ordered scene-id table both registries are
  built on (duplicate and unknown ids, host-side id checks);
* ``OutputSetPool`` keeps the service-owned output sets, keyed by shape, so
  steady-state renders allocate nothing.
"""

from __future__ import annotations

from collections.abc import Callable, Hashable, Iterable
from dataclasses import dataclass
from typing import Generic, TypeVar

import torch

from .contracts import ensure_tensor

T = TypeVar("T")


@dataclass(frozen=True)
class TensorField:
    """One tensor of a scene: attribute name, dims after the leading
    Gaussian-count dim, dtype; ``free_leading`` lets the leading dim define
    the count instead of being checked against it; ``optional`` fields may
    be None."""

    name: str
    trailing: tuple[int | None, ...]
    dtype: torch.dtype
    free_leading: bool = False
    optional: bool = False


def check_fields(owner: object, fields: Iterable[TensorField], count: int, *, device: torch.device,
                 require_cuda: bool) -> None:
    """Validate every tensor of ``owner`` named in ``fields`` (type, device,
    dtype, shape, contiguity) with the boundary's standard messages."""
    for field in fields:
        tensor = getattr(owner, field.name)
        if tensor is None and field.optional:
            continue
        leading = None if field.free_leading else count
        ensure_tensor(tensor, name=field.name, shape=(leading, *field.trailing), dtype=field.dtype,
                      device=device, require_cuda=require_cuda)


class ServiceLifecycle:
    """Device resolution and the initialise-before-use guard of one service."""

    def __init__(self, owner: str, allow_cpu: bool) -> None:
        self.owner = owner
        self.allow_cpu = allow_cpu
        self.device: torch.device | None = None
        self.ready = False

    @property
    def require_cuda(self) -> bool:
        return not self.allow_cpu

    def start(self, device: torch.device | str) -> torch.device:
        resolved = torch.device(device)
        if resolved.type == "cuda" and resolved.index is None:
            resolved = torch.device("cuda", torch.cuda.current_device())
        if resolved.type != "cuda" and not self.allow_cpu:
            raise ValueError(f"{self.owner} requires a CUDA device; got {resolved}.")
        self.device = resolved
        return resolved

    def check(self) -> torch.device:
        if not self.ready or self.device is None:
            raise RuntimeError(f"{self.owner}.initialize(stage, device) must be called first.")
        return self.device


class SceneTable(Generic[T]):
    """Insertion-ordered scene id -> entry.

    ``noun`` names an entry in messages ("scene" / "LiDAR scene"), so the
    camera and LiDAR registries raise the reference's exact texts."""

    def __init__(self, noun: str) -> None:
        self._noun = noun
        self._entries: dict[int, T] = {}

    def __contains__(self, scene_id: int) -> bool:
        return scene_id in self._entries

    def __len__(self) -> int:
        return len(self._entries)

    @property
    def ids(self) -> tuple[int, ...]:
        return tuple(self._entries)

    def values(self) -> list[T]:
        return list(self._entries.values())

    def insert(self, scene_id: int, entry: T) -> None:
        if scene_id in self._entries:
            raise ValueError(f"{self._noun[0].upper()}{self._noun[1:]} {scene_id} is already registered.")
        self._entries[scene_id] = entry

    def lookup(self, scene_id: int) -> T:
        if scene_id not in self._entries:
            raise ValueError(f"Unregistered {self._noun} ID: {scene_id}.")
        return self._entries[scene_id]

    def replace(self, scene_id: int, entry: T) -> None:
        self.lookup(scene_id)
        self._entries[scene_id] = entry

    def check_host_ids(self, scene_ids: torch.Tensor) -> None:
        """Host-side check that every id in a CPU tensor is registered (the
        CUDA path never reads ids back; its kernels mark unknown ids)."""
        if scene_ids.device.type != "cpu":
            raise ValueError(f"Host {self._noun}-ID validation accepts CPU tensors only.")
        unknown = sorted(set(scene_ids.tolist()).difference(self._entries))
        if unknown:
            raise ValueError(f"Unregistered {self._noun} ID(s): {[int(v) for v in unknown]}.")


class OutputSetPool:
    """Service-owned output sets by shape key, created once by ``factory``."""

    def __init__(self, factory: Callable[[Hashable], dict[str, torch.Tensor]],
                 still_valid: Callable[[dict[str, torch.Tensor]], bool] | None = None) -> None:
        self._factory = factory
        self._still_valid = still_valid
        self._sets: dict[Hashable, dict[str, torch.Tensor]] = {}

    def get(self, key: Hashable) -> dict[str, torch.Tensor]:
        found = self._sets.get(key)
        if found is None or (self._still_valid is not None and not self._still_valid(found)):
            found = self._factory(key)
            self._sets[key] = found
        return found

    def clear(self) -> None:
        self._sets.clear()
