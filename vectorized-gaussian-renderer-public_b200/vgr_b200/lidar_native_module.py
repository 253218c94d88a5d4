"""Drop-in LiDAR native module with the reference extension's function surface.

The reference loads a PyTorch extension exporting ``sort_temp_bytes``,
``build_scene_lbvh``, ``pack_scene_descriptor`` and ``render_lidar``
(src/isaacsim_gaussian_renderer/native/lidar_renderer.cpp:62-216) and
injects it into its backend through ``CudaLidarBackend(native_module=...)``.
The functions below accept the same tensor lists and scalars, perform the
same contract checks (lidar_renderer.cpp:62-200, raising RuntimeError like
TORCH_CHECK) and run the B200 kernels of libvgr_b200.so on the current
PyTorch CUDA stream.

The acceleration structure differs from the reference's (planar surfel
records in Morton order and a Karras radix tree over packet leaves with both
child boxes per node, instead of a complete binary tree of node bounds), so
it cannot live in the caller's ``sorted_indices``/``node_bounds`` tensors.
Each scene's structure is kept in a private device buffer tied to the
caller's ``node_bounds`` tensor (released with it).  The reference's backend
always calls ``build_scene_lbvh`` and then ``pack_scene_descriptor`` for a
scene (cuda_lidar_backend.py:315-366); the build needs the opacities,
semantic ids and optional attributes that only the pack receives, so
``build_scene_lbvh`` validates and records the build parameters and
``pack_scene_descriptor`` runs the build and writes the descriptor row.
Descriptor rows keep the reference shape ([S,14] int64).
"""

from __future__ import annotations

import weakref
from dataclasses import dataclass
from typing import Sequence

import torch

from . import _native
from .cuda_lidar_backend import RayOrder
from ._native_signatures import (
    LIDAR_COUNTERS,
    LIDAR_DESCRIPTOR_BYTES,
    VgrLidarInputs,
    VgrLidarOptions,
    VgrLidarOutputs,
    VgrLidarScene,
)

DESCRIPTOR_COLUMNS = 14

# Trace order of the last direction tensor rendered (see cuda_lidar_backend.RayOrder).
_RAY_ORDER = RayOrder()


def _check(cond: bool, message: str) -> None:
    if not cond:
        raise RuntimeError(message)


def _check_group(tensors: Sequence[torch.Tensor], name: str, expected: int) -> None:
    _check(len(tensors) == expected, f"{name} must contain {expected} tensors")
    for index, tensor in enumerate(tensors):
        _check(isinstance(tensor, torch.Tensor), f"{name}[{index}] must be a tensor")
        _check(tensor.is_cuda, f"{name}[{index}] must be a CUDA tensor")
        _check(tensor.is_contiguous(), f"{name}[{index}] must be contiguous")


def _ptr(tensor: torch.Tensor | None) -> int | None:
    return None if tensor is None or tensor.numel() == 0 else tensor.data_ptr()


def _stream(device: torch.device) -> int:
    return torch.cuda.current_stream(device).cuda_stream


@dataclass
class _Pending:
    packet: int
    support_sigma: float
    planarity_ratio_max: float
    count: int
    owner: "weakref.ref[torch.Tensor]"
    accel: torch.Tensor | None = None


# id(node_bounds) -> its scene's acceleration; the entry is dropped when the
# caller's node_bounds tensor is released.
_acceleration: dict[int, _Pending] = {}


def _lookup(node_bounds: torch.Tensor) -> _Pending | None:
    entry = _acceleration.get(id(node_bounds))
    return entry if entry is not None and entry.owner() is node_bounds else None


def sort_temp_bytes(num_items: int) -> int:
    """Temporary bytes of the Morton sort (lidar_renderer.cpp:62-65).  The
    B200 build keeps its sort scratch inside the per-scene structure, so a
    small buffer suffices; the size is positive for the caller's allocation."""
    _check(num_items > 0, "num_items must be positive")
    return 256


def build_scene_lbvh(
    scene: Sequence[torch.Tensor],
    build: Sequence[torch.Tensor],
    packet_size: int,
    leaf_count: int,
    leaf_capacity: int,
    support_sigma: float,
    planarity_ratio_max: float,
) -> None:
    """Contract checks of lidar_renderer.cpp:67-108; the build itself runs in
    pack_scene_descriptor, which receives the remaining scene attributes."""
    _check_group(scene, "scene", 3)
    _check_group(build, "build", 7)
    _check(packet_size in (8, 16), "packet_size must be 8 or 16")
    _check(leaf_count > 0 and leaf_capacity >= leaf_count, "invalid leaf counts")
    _check((leaf_capacity & (leaf_capacity - 1)) == 0, "leaf_capacity must be a power of two")
    _check(support_sigma > 0.0, "support_sigma must be positive")
    _check(0.0 < planarity_ratio_max <= 1.0, "planarity_ratio_max must be in (0, 1]")
    means, scales, rotations = scene
    count = means.size(0)
    _check(means.dtype == torch.float32, "means must be float32")
    _check(scales.dtype == torch.float32, "scales must be float32")
    _check(rotations.dtype == torch.float32, "rotations must be float32")
    _check(tuple(means.shape) == (count, 3), "means shape")
    _check(tuple(scales.shape) == (count, 3), "scales shape")
    _check(tuple(rotations.shape) == (count, 4), "rotations shape")
    _check(build[0].numel() == count, "keys_in size")
    _check(build[1].numel() == count, "keys_out size")
    _check(build[2].numel() == count, "indices_in size")
    _check(build[3].numel() == count, "sorted_indices size")
    _check(tuple(build[5].shape) == (2, 3), "scene_bounds shape")
    _check(tuple(build[6].shape) == (2 * leaf_capacity - 1, 6), "node_bounds shape")
    node_bounds = build[6]
    entry = _lookup(node_bounds)
    if entry is None or entry.count != count or entry.packet != packet_size:
        key = id(node_bounds)
        entry = _Pending(packet_size, support_sigma, planarity_ratio_max, count, weakref.ref(node_bounds))
        _acceleration[key] = entry
        weakref.finalize(node_bounds, _acceleration.pop, key, None)
    entry.support_sigma = support_sigma
    entry.planarity_ratio_max = planarity_ratio_max


def pack_scene_descriptor(
    descriptors: torch.Tensor,
    slot: int,
    scene_id: int,
    scene: Sequence[torch.Tensor],
    leaf_count: int,
    leaf_capacity: int,
) -> None:
    """Build the scene's structure and write descriptor row ``slot``
    (lidar_renderer.cpp:110-131)."""
    _check(descriptors.is_cuda and descriptors.is_contiguous(), "descriptors must be a contiguous CUDA tensor")
    _check_group(scene, "scene", 9)
    _check(descriptors.dtype == torch.int64, "descriptors must be int64")
    _check(descriptors.dim() == 2 and descriptors.size(1) == DESCRIPTOR_COLUMNS, "descriptors shape")
    _check(0 <= slot < descriptors.size(0), "descriptor slot out of range")
    _check(leaf_count > 0 and leaf_capacity >= leaf_count, "invalid leaf metadata")
    means, scales, rotations, opacities, semantic_ids, reflectivity, confidence, _sorted, node_bounds = scene
    entry = _lookup(node_bounds)
    _check(entry is not None, "pack_scene_descriptor needs build_scene_lbvh of the same scene first")
    count = means.size(0)
    _check(entry.count == count, "scene changed size since build_scene_lbvh")
    _check(opacities.dtype == torch.float32 and opacities.numel() == count, "opacities shape")
    _check(semantic_ids.dtype == torch.int64 and semantic_ids.numel() == count, "semantic_ids shape")
    lib = _native.load_library()
    device = means.device
    if entry.accel is None:
        nbytes = _native.check_size(lib.vgr_lidar_sort_temp_bytes(count, entry.packet), "lidar accel")
        entry.accel = torch.empty((nbytes,), dtype=torch.uint8, device=device)
    native_scene = VgrLidarScene(
        means=means.data_ptr(),
        scales=scales.data_ptr(),
        rotations=rotations.data_ptr(),
        opacities=opacities.data_ptr(),
        semantic_ids=semantic_ids.data_ptr(),
        reflectivity=_ptr(reflectivity),
        surface_confidence=_ptr(confidence),
        count=count,
    )
    with torch.cuda.device(device):
        stream = _stream(device)
        _native.check(
            lib.vgr_lidar_build_scene_lbvh(
                native_scene, entry.packet, entry.support_sigma, entry.planarity_ratio_max,
                entry.accel.data_ptr(), entry.accel.numel(), stream,
            ),
            "build_scene_lbvh",
        )
        _native.check(
            lib.vgr_lidar_pack_scene_descriptor(
                descriptors.data_ptr(), descriptors.size(0), slot, scene_id, entry.accel.data_ptr(),
                count, entry.packet, stream,
            ),
            "pack_scene_descriptor",
        )


def render_lidar(
    descriptors: torch.Tensor,
    scene_count: int,
    inputs: Sequence[torch.Tensor],
    outputs: Sequence[torch.Tensor],
    counters: torch.Tensor,
    returns: int,
    packet_size: int,
    near_plane_m: float,
    far_plane_m: float,
    support_sigma: float,
    detection_threshold: float,
    planarity_ratio_max: float,
    min_incidence_cos: float,
    cluster_abs_m: float,
    cluster_relative: float,
    fallback_reflectivity: float,
    direction_norm_tolerance: float,
    semantic_slots: int,
) -> None:
    """Trace one LiDAR invocation (lidar_renderer.cpp:133-210)."""
    _check(descriptors.is_cuda and descriptors.is_contiguous(), "descriptors must be a contiguous CUDA tensor")
    _check(counters.is_cuda and counters.is_contiguous(), "counters must be a contiguous CUDA tensor")
    _check_group(inputs, "inputs", 6)
    _check_group(outputs, "outputs", 7)
    _check(0 < scene_count <= descriptors.size(0), "invalid scene_count")
    _check(returns in (1, 2), "returns must be 1 or 2")
    _check(packet_size in (8, 16), "packet_size must be 8 or 16")
    _check(near_plane_m > 0.0 and far_plane_m > near_plane_m, "invalid range planes")
    _check(support_sigma > 0.0, "support_sigma must be positive")
    _check(0.0 < detection_threshold <= 1.0, "invalid threshold")
    _check(0.0 < planarity_ratio_max <= 1.0, "invalid planarity")
    _check(0.0 < min_incidence_cos <= 1.0, "invalid incidence")
    _check(cluster_abs_m >= 0.0 and cluster_relative >= 0.0, "invalid cluster")
    _check(0.0 <= fallback_reflectivity <= 1.0, "invalid reflectivity")
    _check(0.0 < direction_norm_tolerance < 1.0, "direction tolerance must be in (0, 1)")
    _check(0 < semantic_slots <= 32, "semantic_slots must be in [1, 32]")
    _check(counters.dtype == torch.int64 and counters.numel() == LIDAR_COUNTERS, "counters shape")
    directions, times, sensor_to_world, scene_to_world, scene_ids, active = inputs
    rays = directions.size(0)
    batch = sensor_to_world.size(0)
    _check(tuple(directions.shape) == (rays, 3), "ray directions shape")
    _check(directions.dtype == torch.float32, "ray directions dtype")
    _check(times.size(0) == rays, "time offsets shape")
    _check(times.dtype in (torch.int32, torch.int64), "time offsets dtype")
    _check(tuple(sensor_to_world.shape) == (batch, 4, 4), "sensor transforms shape")
    _check(tuple(scene_to_world.shape) == (batch, 4, 4), "scene transforms shape")
    _check(tuple(scene_ids.shape) == (batch,), "scene IDs shape")
    _check(active.dim() == 1, "active IDs shape")
    rng, position, intensity, semantic, valid, time_out, count = outputs
    _check(tuple(rng.shape) == (batch, rays, returns), "range shape")
    _check(tuple(position.shape) == (batch, rays, returns, 3), "position shape")
    _check(tuple(intensity.shape) == (batch, rays, returns), "intensity shape")
    _check(tuple(semantic.shape) == (batch, rays, returns), "semantic shape")
    _check(tuple(valid.shape) == (batch, rays, returns), "valid shape")
    _check(tuple(time_out.shape) == (batch, rays, returns), "time output shape")
    _check(tuple(count.shape) == (batch, rays), "count shape")
    lib = _native.load_library()
    native_inputs = VgrLidarInputs(
        ray_directions=directions.data_ptr(),
        rays=rays,
        time_offsets=times.data_ptr(),
        time_offsets_are_int64=int(times.dtype == torch.int64),
        sensor_to_world=sensor_to_world.data_ptr(),
        scene_to_world=scene_to_world.data_ptr(),
        scene_ids=scene_ids.data_ptr(),
        batch=batch,
        active_sensor_ids=_ptr(active),
        active_count=active.numel(),
        ray_order=_RAY_ORDER(directions).data_ptr(),
    )
    native_outputs = VgrLidarOutputs(
        range_m=rng.data_ptr(),
        position_world_m=position.data_ptr(),
        intensity=intensity.data_ptr(),
        semantic_id=semantic.data_ptr(),
        valid=valid.data_ptr(),
        time_offset_ns=time_out.data_ptr(),
        return_count=count.data_ptr(),
    )
    options = VgrLidarOptions(
        returns=returns,
        semantic_slots=semantic_slots,
        near_plane_m=near_plane_m,
        far_plane_m=far_plane_m,
        support_sigma=support_sigma,
        detection_threshold=detection_threshold,
        planarity_ratio_max=planarity_ratio_max,
        min_incidence_cos=min_incidence_cos,
        cluster_abs_m=cluster_abs_m,
        cluster_relative=cluster_relative,
        fallback_reflectivity=fallback_reflectivity,
        direction_norm_tolerance=direction_norm_tolerance,
    )
    device = directions.device
    with torch.cuda.device(device):
        _native.check(
            lib.vgr_render_lidar(
                descriptors.data_ptr(), scene_count, native_inputs, native_outputs, counters.data_ptr(),
                options, _stream(device),
            ),
            "render_lidar",
        )


class NativeLidarModule:
    """Object form of this module, for ``native_module=`` injection."""

    sort_temp_bytes = staticmethod(sort_temp_bytes)
    build_scene_lbvh = staticmethod(build_scene_lbvh)
    pack_scene_descriptor = staticmethod(pack_scene_descriptor)
    render_lidar = staticmethod(render_lidar)


def load_lidar_extension() -> NativeLidarModule:
    """Counterpart of the reference ``lidar_native_loader`` entry point."""
    _native.load_library()
    _check(LIDAR_DESCRIPTOR_BYTES <= DESCRIPTOR_COLUMNS * 8, "descriptor rows are too narrow")
    return NativeLidarModule()
