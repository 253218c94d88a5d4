"""Drop-in native module with the reference extension's function surface.

The reference loads a PyTorch extension exporting ``render``,
``sort_temp_bytes``, ``radix_sort_double_buffer_temp_bytes``,
``precompute_covariances``, ``prepare_chunked_active_ids`` and
``aggregate_chunk_counters`` (src/isaacsim_gaussian_renderer/native/
renderer.cpp:312-337) and injects it into its backend through
``CustomCudaBackend(native_module=...)`` (cuda_backend.py:123-124).  The
functions below accept the same tensor lists and scalars, perform the same
contract checks (renderer.cpp:9-25,214-283 and renderer_cuda.cu:2561-2730,
raising RuntimeError like TORCH_CHECK) and forward raw pointers to the C ABI
of libvgr_b200.so on the current PyTorch CUDA stream.

``render`` keeps the reference's 24-tensor workspace: keys/values double
buffers, tile ranges and counters are used in place; the visible-record
structure-of-arrays tensors are filled as mirrors; the 48-byte projected
records and the frame scratch live in ``sort_temp``, whose size this
module reports through the two temp-bytes queries.
"""

from __future__ import annotations

import math
from typing import Sequence

import torch

from . import _native

SCENE_TENSORS = 7
CAMERA_TENSORS = 5
OUTPUT_TENSORS = 4
WORKSPACE_TENSORS = 24

# Workspace order of the reference (renderer_cuda.cu:73-98).
(
    K_VISIBLE_MEANS2D,
    K_VISIBLE_CONICS,
    K_VISIBLE_DEPTHS,
    K_VISIBLE_OPACITIES,
    K_VISIBLE_CAMERA_IDS,
    K_VISIBLE_GAUSSIAN_IDS,
    K_VISIBLE_RADII,
    K_KEYS_IN,
    K_KEYS_OUT,
    K_VALUES_IN,
    K_VALUES_OUT,
    K_TILE_STARTS,
    K_TILE_ENDS,
    K_COUNTERS,
    K_SORT_TEMP,
) = range(15)
K_VISIBLE_RAY_PRECISIONS = 22
K_VISIBLE_RAY_PRECISION_MEANS = 23


def _check(cond: bool, *message: object) -> None:
    if not cond:
        raise RuntimeError("".join(str(part) for part in message))


def _check_group(tensors: Sequence[torch.Tensor], name: str, expected: int) -> None:
    _check(
        len(tensors) == expected,
        name,
        " must contain ",
        expected,
        " tensors, got ",
        len(tensors),
    )
    for index, tensor in enumerate(tensors):
        _check(tensor.is_cuda, name, "[", index, "] must be CUDA-resident")
        _check(tensor.is_contiguous(), name, "[", index, "] must be contiguous")


def _check_dtype(tensor: torch.Tensor, dtype: torch.dtype, name: str) -> None:
    _check(
        tensor.dtype == dtype,
        name,
        " has dtype ",
        tensor.dtype,
        ", expected ",
        dtype,
    )


def _ptr(tensor: torch.Tensor | None) -> int | None:
    if tensor is None or tensor.numel() == 0:
        return None
    return tensor.data_ptr()


def _stream(device: torch.device) -> int:
    return torch.cuda.current_stream(device).cuda_stream


def sort_temp_bytes(num_items: int, num_segments: int) -> int:
    """Scratch bytes for the deterministic path (renderer.cpp:76-81)."""
    _check(num_items > 0, "num_items must be positive")
    _check(num_segments > 0, "num_segments must be positive")
    lib = _native.load_library()
    return _native.check_size(lib.vgr_sort_temp_bytes(num_items, num_segments), "sort_temp_bytes")


def radix_sort_double_buffer_temp_bytes(num_items: int, num_segments: int) -> int:
    """Scratch bytes for the double-buffer path (renderer.cpp:83-90)."""
    _check(num_items > 0, "num_items must be positive")
    _check(num_segments > 0, "num_segments must be positive")
    lib = _native.load_library()
    return _native.check_size(
        lib.vgr_radix_sort_double_buffer_temp_bytes(num_items, num_segments),
        "radix_sort_double_buffer_temp_bytes",
    )


def precompute_covariances(
    scales: torch.Tensor,
    rotations: torch.Tensor,
    covariances: torch.Tensor,
) -> None:
    """Sigma = R S S^T R^T upper triangle (renderer.cpp:92-131)."""
    _check(scales.is_cuda, "scales must be CUDA-resident")
    _check(rotations.is_cuda, "rotations must be CUDA-resident")
    _check(covariances.is_cuda, "covariances must be CUDA-resident")
    _check(
        scales.device == rotations.device and scales.device == covariances.device,
        "scales, rotations, and covariances must share a CUDA device",
    )
    _check(scales.is_contiguous(), "scales must be contiguous")
    _check(rotations.is_contiguous(), "rotations must be contiguous")
    _check(covariances.is_contiguous(), "covariances must be contiguous")
    _check(scales.dtype == torch.float32, "scales must be float32")
    _check(rotations.dtype == torch.float32, "rotations must be float32")
    _check(covariances.dtype == torch.float32, "covariances must be float32")
    _check(scales.dim() == 2 and scales.size(1) == 3, "scales must have shape [G, 3]")
    _check(rotations.dim() == 2 and rotations.size(1) == 4, "rotations must have shape [G, 4]")
    _check(
        covariances.dim() == 2 and covariances.size(1) == 6,
        "covariances must have shape [G, 6]",
    )
    _check(
        scales.size(0) == rotations.size(0) and scales.size(0) == covariances.size(0),
        "scales, rotations, and covariances must share G",
    )
    lib = _native.load_library()
    with torch.cuda.device(scales.device):
        _native.check(
            lib.vgr_precompute_covariances(
                _ptr(scales),
                _ptr(rotations),
                scales.size(0),
                _ptr(covariances),
                _stream(scales.device),
            ),
            "precompute_covariances",
        )


def prepare_chunked_active_ids(
    active_camera_ids: torch.Tensor,
    active_mask: torch.Tensor,
    chunk_active_ids: torch.Tensor,
    logical_batch: int,
    physical_batch: int,
) -> None:
    """Padded chunk-local active ids on the device (renderer.cpp:133-181)."""
    _check(
        active_camera_ids.is_cuda and active_mask.is_cuda and chunk_active_ids.is_cuda,
        "chunked active-ID tensors must be CUDA-resident",
    )
    _check(
        active_camera_ids.is_contiguous()
        and active_mask.is_contiguous()
        and chunk_active_ids.is_contiguous(),
        "chunked active-ID tensors must be contiguous",
    )
    _check(
        active_camera_ids.device == active_mask.device
        and active_camera_ids.device == chunk_active_ids.device,
        "chunked active-ID tensors must share a device",
    )
    _check(active_camera_ids.dtype == torch.int64, "active_camera_ids must be int64")
    _check(active_mask.dtype == torch.int32, "active_mask must be int32")
    _check(chunk_active_ids.dtype == torch.int64, "chunk_active_ids must be int64")
    _check(
        active_camera_ids.dim() == 1 and active_mask.dim() == 1 and chunk_active_ids.dim() == 2,
        "invalid chunked active-ID tensor ranks",
    )
    _check(logical_batch > 0 and physical_batch > 0, "logical and physical batches must be positive")
    lib = _native.load_library()
    with torch.cuda.device(active_camera_ids.device):
        _native.check(
            lib.vgr_prepare_chunked_active_ids(
                _ptr(active_camera_ids),
                active_camera_ids.numel(),
                _ptr(active_mask),
                active_mask.numel(),
                _ptr(chunk_active_ids),
                chunk_active_ids.size(0),
                chunk_active_ids.size(1),
                logical_batch,
                physical_batch,
                _stream(active_camera_ids.device),
            ),
            "prepare_chunked_active_ids",
        )


def aggregate_chunk_counters(
    chunk_counters: torch.Tensor,
    counters: torch.Tensor,
    physical_capacity_counters: torch.Tensor,
    chunk_count: int,
) -> None:
    """Reduce per-chunk counters to logical totals and maxima (renderer.cpp:183-212)."""
    _check(
        chunk_counters.is_cuda and counters.is_cuda and physical_capacity_counters.is_cuda,
        "chunk counters must be CUDA-resident",
    )
    _check(
        chunk_counters.is_contiguous()
        and counters.is_contiguous()
        and physical_capacity_counters.is_contiguous(),
        "chunk counters must be contiguous",
    )
    _check(
        chunk_counters.dtype == torch.int64
        and counters.dtype == torch.int64
        and physical_capacity_counters.dtype == torch.int64,
        "chunk counters must be int64",
    )
    _check(
        chunk_counters.dim() == 2
        and chunk_counters.size(1) >= 5
        and counters.numel() >= 5
        and physical_capacity_counters.numel() >= 5,
        "chunk counters must have shape [N, >=5] and outputs >=5",
    )
    _check(
        0 < chunk_count <= chunk_counters.size(0),
        "chunk_count exceeds the counter workspace",
    )
    lib = _native.load_library()
    with torch.cuda.device(chunk_counters.device):
        _native.check(
            lib.vgr_aggregate_chunk_counters(
                _ptr(chunk_counters),
                chunk_counters.size(0),
                chunk_counters.size(1),
                _ptr(counters),
                _ptr(physical_capacity_counters),
                chunk_count,
                _stream(chunk_counters.device),
            ),
            "aggregate_chunk_counters",
        )


_private_scratch: dict[tuple[torch.device, int], torch.Tensor] = {}
_private_buffers: dict[tuple, torch.Tensor] = {}


def _private_buffer(key: tuple, numel: int, dtype: torch.dtype, device: torch.device) -> torch.Tensor:
    """A cached device buffer of at least ``numel`` elements."""
    buf = _private_buffers.get(key)
    if buf is None or buf.numel() < numel or buf.dtype != dtype:
        buf = torch.empty((max(numel, 1),), dtype=dtype, device=device)
        _private_buffers[key] = buf
    return buf


def _scratch_and_records(
    sort_temp: torch.Tensor,
    need: int,
    visible_capacity: int,
    intersection_capacity: int,
    record_bytes: int = _native.RECORD_BYTES,
) -> tuple[torch.Tensor, int, int, int]:
    """Carve (scratch, records) from sort_temp, or from a cached private buffer.

    A visible record covers at least one tile, so min(visible, intersection
    capacity) records always suffice.  record_bytes is the storage per visible
    record (twice RECORD_BYTES in exact-ray mode, whose extension records
    follow the records).
    Returns (storage, scratch_bytes, records_offset, record_capacity).
    """
    records = max(1, min(visible_capacity, intersection_capacity))
    aligned = (need + 255) // 256 * 256
    available = sort_temp.numel() - aligned
    if available >= records * record_bytes:
        return sort_temp, need, aligned, records
    visible_capacity = records
    size = aligned + visible_capacity * record_bytes
    key = (sort_temp.device, size)
    storage = _private_scratch.get(key)
    if storage is None:
        _private_scratch.clear()
        storage = torch.empty(size, dtype=torch.uint8, device=sort_temp.device)
        _private_scratch[key] = storage
    return storage, need, aligned, visible_capacity


def render(
    scene: Sequence[torch.Tensor],
    cameras: Sequence[torch.Tensor],
    outputs: Sequence[torch.Tensor],
    workspace: Sequence[torch.Tensor],
    height: int,
    width: int,
    max_scene_gaussians: int,
    near_plane: float,
    far_plane: float,
    gaussian_support_sigma: float,
    covariance_epsilon: float,
    antialiased: bool,
    semantic_min_alpha: float,
    ray_gaussian_evaluation: bool,
    tile_size: int,
    depth_bucket_count: int,
    depth_bucket_group_size: int,
    compact_projection_cache: bool,
    materialize_projected_records: bool,
    reuse_projection: bool,
    output_srgb: bool,
    deterministic: bool,
    full_sensor_output: bool,
    fixed_capacity_sort: bool,
) -> int:
    """Project, order and composite one batch (renderer.cpp:214-310).

    Returns the sorted-buffer selector: 1 when keys_out/values_out hold the
    sorted lists, 0 when keys_in/values_in do.
    """
    _check_group(scene, "scene", SCENE_TENSORS)
    _check_group(cameras, "cameras", CAMERA_TENSORS)
    _check_group(outputs, "outputs", OUTPUT_TENSORS)
    _check_group(workspace, "workspace", WORKSPACE_TENSORS)
    _check(height > 0 and width > 0, "height and width must be positive")
    _check(max_scene_gaussians > 0, "max_scene_gaussians must be positive")
    _check(near_plane > 0.0, "near_plane must be positive")
    _check(far_plane > near_plane, "far_plane must be greater than near_plane")
    _check(gaussian_support_sigma > 0.0, "gaussian_support_sigma must be positive")
    _check(
        math.isfinite(covariance_epsilon) and covariance_epsilon >= 0.0,
        "covariance_epsilon must be finite and non-negative",
    )
    _check(
        math.isfinite(semantic_min_alpha) and 0.0 <= semantic_min_alpha <= 1.0,
        "semantic_min_alpha must be finite and in [0, 1]",
    )
    _check(
        0 < tile_size <= 16 and (tile_size & (tile_size - 1)) == 0,
        "tile_size must be a power of two in [1, 16]",
    )
    _check(depth_bucket_count > 0, "depth_bucket_count must be positive")
    _check(depth_bucket_group_size > 0, "depth_bucket_group_size must be positive")
    _check(
        not compact_projection_cache or tile_size == 1,
        "compact_projection_cache requires tile_size=1",
    )
    _check(
        not compact_projection_cache or not ray_gaussian_evaluation,
        "compact_projection_cache supports only screen-space evaluation",
    )
    _check(
        not antialiased or not ray_gaussian_evaluation,
        "antialiased rasterization is incompatible with exact-ray evaluation",
    )
    _check(
        not compact_projection_cache or not deterministic,
        "compact_projection_cache currently requires deterministic=false",
    )
    _check(
        not materialize_projected_records or compact_projection_cache,
        "materialize_projected_records requires compact_projection_cache",
    )
    _check(
        not fixed_capacity_sort or not deterministic,
        "fixed_capacity_sort applies only to the nondeterministic path",
    )

    means, covariances, opacities, features, semantic_ids, registered, offsets = scene
    viewmats, intrinsics, env_xforms, camera_scene_ids, active_ids = cameras
    rgb, depth, alpha, semantic = outputs
    for tensor, dtype, name in (
        (means, torch.float32, "means"),
        (covariances, torch.float32, "covariances"),
        (opacities, torch.float32, "opacities"),
        (features, torch.float32, "features"),
        (semantic_ids, torch.int64, "semantic_ids"),
        (registered, torch.int64, "registered_scene_ids"),
        (offsets, torch.int64, "scene_offsets"),
        (viewmats, torch.float32, "viewmats"),
        (intrinsics, torch.float32, "intrinsics"),
        (env_xforms, torch.float32, "env_xforms"),
        (camera_scene_ids, torch.int64, "camera_scene_ids"),
        (active_ids, torch.int64, "active_camera_ids"),
        (rgb, torch.float32, "rgb"),
        (depth, torch.float32, "depth"),
        (alpha, torch.float32, "alpha"),
        (semantic, torch.int64, "semantic"),
        (workspace[K_KEYS_IN], torch.uint64, "keys_in"),
        (workspace[K_KEYS_OUT], torch.uint64, "keys_out"),
        (workspace[K_VALUES_IN], torch.int32, "values_in"),
        (workspace[K_VALUES_OUT], torch.int32, "values_out"),
        (workspace[K_TILE_STARTS], torch.int32, "tile_starts"),
        (workspace[K_TILE_ENDS], torch.int32, "tile_ends"),
        (workspace[K_COUNTERS], torch.int64, "counters"),
        (workspace[K_SORT_TEMP], torch.uint8, "sort_temp"),
    ):
        _check_dtype(tensor, dtype, name)
    batch = viewmats.size(0)
    active_count = active_ids.numel() if active_ids.numel() else batch
    feature_width = features.size(1)
    _check(feature_width >= 3, "features must provide at least RGB channels")
    _check(env_xforms.size(0) >= batch, "env_xforms must provide one transform per camera")
    _check(
        workspace[K_TILE_STARTS].numel() == workspace[K_TILE_ENDS].numel(),
        "tile start and end workspaces must have the same capacity",
    )
    _check(workspace[K_COUNTERS].numel() >= 5, "counters workspace must contain at least five int64 values")

    # Exact-ray mode bins 16-pixel tiles as 32-pixel tiles (renderer_cuda.cu:2670-2676);
    # dense mode (tile_size 1) runs on 16-pixel tiles with its depth cutoff.
    _check(not (tile_size == 1 and ray_gaussian_evaluation),
           "dense mode (tile_size=1) renders screen-space evaluation only in this build")
    bin_tile = 32 if ray_gaussian_evaluation and tile_size == 16 else 16 if tile_size == 1 else tile_size
    tiles_x = -(-width // bin_tile)
    tiles_y = -(-height // bin_tile)
    global_tiles = batch * tiles_x * tiles_y
    visible_capacity = workspace[K_VISIBLE_DEPTHS].numel()
    intersection_capacity = workspace[K_KEYS_IN].numel()
    _check(visible_capacity > 0, "visible capacity must be positive")
    _check(intersection_capacity > 0, "intersection capacity must be positive")
    if ray_gaussian_evaluation:
        # Workspace contract of the exact-ray path (renderer_cuda.cu:2721-2730);
        # this build keeps the precision terms in its own extension records.
        _check_dtype(workspace[K_VISIBLE_RAY_PRECISIONS], torch.float32, "visible_ray_precisions")
        _check_dtype(workspace[K_VISIBLE_RAY_PRECISION_MEANS], torch.float32, "visible_ray_precision_means")
        _check(workspace[K_VISIBLE_RAY_PRECISIONS].numel() >= visible_capacity * 6,
               "visible ray-precision workspace is too small")
        _check(workspace[K_VISIBLE_RAY_PRECISION_MEANS].numel() >= visible_capacity * 4,
               "visible ray precision-mean workspace is too small")

    lib = _native.load_library()
    need = _native.check_size(
        lib.vgr_render_scratch_bytes(
            intersection_capacity,
            active_count * max_scene_gaussians,
            max(global_tiles, 1),
            active_count,
        ),
        "render scratch",
    )
    storage, scratch_bytes, records_offset, record_capacity = _scratch_and_records(
        workspace[K_SORT_TEMP], need, visible_capacity, intersection_capacity,
        _native.RECORD_BYTES * (2 if ray_gaussian_evaluation else 1),
    )
    mirror = (
        workspace[K_VISIBLE_MEANS2D].numel() >= 2 * record_capacity
        and workspace[K_VISIBLE_CONICS].numel() >= 3 * record_capacity
        and workspace[K_VISIBLE_OPACITIES].numel() >= record_capacity
        and workspace[K_VISIBLE_CAMERA_IDS].numel() >= record_capacity
        and workspace[K_VISIBLE_GAUSSIAN_IDS].numel() >= record_capacity
        and workspace[K_VISIBLE_RADII].numel() >= 2 * record_capacity
    )

    native_scene = _native.VgrScene(
        means=_ptr(means),
        covariances=_ptr(covariances),
        opacities=_ptr(opacities),
        features=_ptr(features),
        feature_width=feature_width,
        semantic_ids=_ptr(semantic_ids),
        registered_scene_ids=_ptr(registered),
        scene_offsets=_ptr(offsets),
        scene_count=registered.numel(),
        gaussian_count=means.size(0),
        max_scene_gaussians=max_scene_gaussians,
    )
    native_cameras = _native.VgrCameras(
        viewmats=_ptr(viewmats),
        intrinsics=_ptr(intrinsics),
        env_xforms=_ptr(env_xforms),
        camera_scene_ids=_ptr(camera_scene_ids),
        active_camera_ids=_ptr(active_ids),
        batch=batch,
        active_count=active_count,
    )
    native_outputs = _native.VgrOutputs(
        rgb=_ptr(rgb),
        depth=_ptr(depth) if full_sensor_output else None,
        alpha=_ptr(alpha) if full_sensor_output else None,
        semantic=_ptr(semantic) if full_sensor_output else None,
    )
    base = storage.data_ptr()
    depth_tau = tile_cutoff = None
    if tile_size == 1:
        # The reference aliases its depth-bucket workspace with sort_temp,
        # which holds this build's records and scratch: private buffers.
        cells = batch * -(-height // _native.DENSE_CELL) * -(-width // _native.DENSE_CELL)
        depth_tau = _private_buffer(("depth_tau", means.device), cells * _native.DENSE_DEPTH_BUCKETS,
                                    torch.float32, means.device)
        tile_cutoff = _private_buffer(("tile_cutoff", means.device), global_tiles, torch.int32, means.device)
    native_workspace = _native.VgrWorkspace(
        records=base + records_offset,
        visible_capacity=record_capacity,
        keys_in=_ptr(workspace[K_KEYS_IN]),
        keys_out=_ptr(workspace[K_KEYS_OUT]),
        values_in=_ptr(workspace[K_VALUES_IN]),
        values_out=_ptr(workspace[K_VALUES_OUT]),
        intersection_capacity=intersection_capacity,
        tile_starts=_ptr(workspace[K_TILE_STARTS]),
        tile_ends=_ptr(workspace[K_TILE_ENDS]),
        tile_capacity=workspace[K_TILE_STARTS].numel(),
        counters=_ptr(workspace[K_COUNTERS]),
        scratch=base,
        scratch_bytes=scratch_bytes,
        visible_means2d=_ptr(workspace[K_VISIBLE_MEANS2D]) if mirror else None,
        visible_conics=_ptr(workspace[K_VISIBLE_CONICS]) if mirror else None,
        visible_depths=_ptr(workspace[K_VISIBLE_DEPTHS]) if mirror else None,
        visible_opacities=_ptr(workspace[K_VISIBLE_OPACITIES]) if mirror else None,
        visible_camera_ids=_ptr(workspace[K_VISIBLE_CAMERA_IDS]) if mirror else None,
        visible_gaussian_ids=_ptr(workspace[K_VISIBLE_GAUSSIAN_IDS]) if mirror else None,
        visible_radii=_ptr(workspace[K_VISIBLE_RADII]) if mirror else None,
        visible_ray_precisions=_ptr(workspace[K_VISIBLE_RAY_PRECISIONS]) if ray_gaussian_evaluation else None,
        visible_ray_precision_means=(_ptr(workspace[K_VISIBLE_RAY_PRECISION_MEANS])
                                     if ray_gaussian_evaluation else None),
        depth_tau=None if depth_tau is None else depth_tau.data_ptr(),
        depth_tau_capacity=0 if depth_tau is None else depth_tau.numel(),
        tile_cutoff=None if tile_cutoff is None else tile_cutoff.data_ptr(),
        tile_cutoff_capacity=0 if tile_cutoff is None else tile_cutoff.numel(),
    )
    options = _native.VgrRenderOptions(
        height=height,
        width=width,
        near_plane=near_plane,
        far_plane=far_plane,
        gaussian_support_sigma=gaussian_support_sigma,
        covariance_epsilon=covariance_epsilon,
        semantic_min_alpha=semantic_min_alpha,
        antialiased=int(bool(antialiased)),
        ray_gaussian_evaluation=int(bool(ray_gaussian_evaluation)),
        tile_size=tile_size,
        output_srgb=int(bool(output_srgb)),
        deterministic=int(bool(deterministic)),
        full_sensor_output=int(bool(full_sensor_output)),
        fixed_capacity_sort=int(bool(fixed_capacity_sort)),
        reuse_projection=int(bool(reuse_projection)),
        compact_projection_cache=int(bool(compact_projection_cache)),
        sh_degree=-1,
        sorted_buffer_hint=1,
    )
    selector = _native._c_i64(1)
    device = means.device
    with torch.cuda.device(device):
        _native.check(
            lib.vgr_render(
                native_scene,
                native_cameras,
                native_outputs,
                native_workspace,
                options,
                _stream(device),
                selector,
            ),
            "render",
        )
    return int(selector.value)


class NativeRendererModule:
    """Object form of this module, for ``native_module=`` injection."""

    sort_temp_bytes = staticmethod(sort_temp_bytes)
    radix_sort_double_buffer_temp_bytes = staticmethod(radix_sort_double_buffer_temp_bytes)
    precompute_covariances = staticmethod(precompute_covariances)
    prepare_chunked_active_ids = staticmethod(prepare_chunked_active_ids)
    aggregate_chunk_counters = staticmethod(aggregate_chunk_counters)
    render = staticmethod(render)


def load_native_extension() -> NativeRendererModule:
    """Counterpart of the reference ``native_loader.load_native_extension``."""
    _native.load_library()
    return NativeRendererModule()
