"""B200 camera backend behind the reference's ``GaussianRendererBackend`` seam.

Drop-in for the reference ``CustomCudaBackend``
(src/isaacsim_gaussian_renderer/cuda_backend.py:63-2231): the same
constructor options, lifecycle, counters (COUNTER_NAMES), bounded adaptive
capacity (grow/retry, then ``RendererCapacityError`` with NaN/-1 outputs),
validated-input reuse without host synchronisation, optional projection
cache, logical -> physical chunking and telemetry properties.

What differs is underneath: one C-ABI call per frame into libvgr_b200.so
(projection + ordered compaction + emission, device-bounded radix sort,
ranges, compositor), with no emitted-count readback, a deterministic order in
every mode, and a workspace of 48-byte packed records instead of the
reference's structure-of-arrays visible tensors (those can be mirrored with
``mirror_reference_workspace=True`` for tools that read them).

``tile_size=1`` (the reference's dense per-pixel path, with or without
``compact_projection_cache``) selects dense mode: 16-pixel tiles whose keys
are culled behind a per-tile optical-thickness depth cutoff, with the images
of the plain path.  ``ray_gaussian_evaluation=True`` selects exact-ray
evaluation.
"""

from __future__ import annotations

import copy
import math
from collections import OrderedDict
from collections.abc import Callable
from typing import Any, Literal, NoReturn

import torch

from . import _native
from .backend import RenderRequest, RenderStats
from .scene import GaussianScene

FULL_SENSOR_OUTPUTS = ("rgb", "depth", "alpha", "semantic_id")
RGB_ONLY_OUTPUTS = ("rgb",)
DEFAULT_GAUSSIAN_SUPPORT_SIGMA = 3.33
COUNTER_NAMES = (
    "visible_gaussians",
    "tile_intersections",
    "visible_overflow",
    "intersection_overflow",
    "active_tiles",
)
DEVICE_STATUS_LOOKBACK_TIMEOUT = 1
_INT32_MAX = 2_147_483_647


def _emitted_sort_key_end_bit(global_tile_capacity: int) -> int:
    """32 + bit width of the largest tile id (renderer_cuda.cu:28-46)."""
    if global_tile_capacity <= 0:
        raise ValueError("Global tile capacity must be positive.")
    if global_tile_capacity > _INT32_MAX:
        raise ValueError("Global tile capacity exceeds the int32 implementation limit.")
    return 32 + (global_tile_capacity - 1).bit_length()


class RendererCapacityError(RuntimeError):
    """Raised when bounded capacity handling cannot produce a valid render."""

    def __init__(self, message: str, *, telemetry: dict[str, Any] | None = None) -> None:
        super().__init__(message)
        self.telemetry = copy.deepcopy(telemetry)


def _default_native_loader():
    from .native_module import load_native_extension

    return load_native_extension()


def _tensor_token(tensor: torch.Tensor) -> tuple[Any, ...]:
    try:
        version: Any = int(tensor._version)
    except RuntimeError:
        # Inference tensors have no version counter: never reuse them.
        version = object()
    return (
        tensor.data_ptr(),
        version,
        tuple(tensor.shape),
        tuple(tensor.stride()),
        tensor.dtype,
        tensor.device,
    )


class CustomCudaBackend:
    def __init__(
        self,
        *,
        max_visible_records: int | None = None,
        max_intersections: int | None = None,
        visible_capacity_per_view: int = 100_000,
        intersections_per_visible: float = 4.0,
        near_plane: float = 0.01,
        far_plane: float = 100.0,
        gaussian_support_sigma: float = DEFAULT_GAUSSIAN_SUPPORT_SIGMA,
        covariance_epsilon: float = 0.3,
        rasterize_mode: Literal["classic", "antialiased"] = "classic",
        semantic_min_alpha: float = 0.01,
        ray_gaussian_evaluation: bool = False,
        tile_size: int = 16,
        depth_bucket_count: int = 4096,
        depth_bucket_group_size: int = 64,
        compact_projection_cache: bool = False,
        materialize_projected_records: bool = False,
        enable_projection_cache: bool = False,
        output_srgb: bool = True,
        deterministic: bool = False,
        fixed_capacity_sort: bool = False,
        max_physical_views: int | None = None,
        adaptive_capacity: bool = True,
        capacity_growth_factor: float = 1.25,
        capacity_headroom: float = 1.25,
        max_capacity_retries: int = 4,
        max_workspace_bytes: int | None = None,
        native_module: Any | None = None,
        native_loader: Callable[[], Any] = _default_native_loader,
        allow_cpu_for_tests: bool = False,
        sh_degree: int | None = None,
        mirror_reference_workspace: bool = False,
        spatial_layout: bool = True,
        persistent_compositor: bool = False,
        composite_shape: int = 2,
    ) -> None:
        if max_visible_records is not None and max_visible_records <= 0:
            raise ValueError("max_visible_records must be positive.")
        if max_intersections is not None and max_intersections <= 0:
            raise ValueError("max_intersections must be positive.")
        if visible_capacity_per_view <= 0:
            raise ValueError("visible_capacity_per_view must be positive.")
        if intersections_per_visible <= 0:
            raise ValueError("intersections_per_visible must be positive.")
        if near_plane <= 0 or far_plane <= near_plane:
            raise ValueError("Expected 0 < near_plane < far_plane.")
        if gaussian_support_sigma <= 0:
            raise ValueError("gaussian_support_sigma must be positive.")
        if not math.isfinite(covariance_epsilon) or covariance_epsilon < 0:
            raise ValueError("covariance_epsilon must be finite and non-negative.")
        if rasterize_mode not in ("classic", "antialiased"):
            raise ValueError("rasterize_mode must be 'classic' or 'antialiased'.")
        if not math.isfinite(semantic_min_alpha) or not 0 <= semantic_min_alpha <= 1:
            raise ValueError("semantic_min_alpha must be finite and in [0, 1].")
        if tile_size <= 0 or tile_size > 16 or tile_size & (tile_size - 1):
            raise ValueError("tile_size must be a power of two in [1, 16].")
        if depth_bucket_count <= 0:
            raise ValueError("depth_bucket_count must be positive.")
        if depth_bucket_group_size <= 0:
            raise ValueError("depth_bucket_group_size must be positive.")
        if compact_projection_cache and tile_size != 1:
            raise ValueError("compact_projection_cache requires tile_size=1.")
        if rasterize_mode == "antialiased" and ray_gaussian_evaluation:
            raise ValueError(
                "rasterize_mode='antialiased' is incompatible with ray_gaussian_evaluation=True."
            )
        if materialize_projected_records and not compact_projection_cache:
            raise ValueError("materialize_projected_records requires compact_projection_cache=True.")
        if fixed_capacity_sort and deterministic:
            raise ValueError(
                "fixed_capacity_sort is only meaningful for the nondeterministic global-radix path."
            )
        if max_physical_views is not None and max_physical_views <= 0:
            raise ValueError("max_physical_views must be positive when set.")
        if max_physical_views is not None and not fixed_capacity_sort:
            raise ValueError(
                "max_physical_views requires fixed_capacity_sort=True so logical chunks never "
                "synchronize on an emitted count."
            )
        if max_physical_views is not None and adaptive_capacity:
            raise ValueError(
                "max_physical_views requires adaptive_capacity=False; physical capacities must be "
                "calibrated and installed before steady-state logical-batch rendering."
            )
        if max_physical_views is not None and enable_projection_cache:
            raise ValueError("max_physical_views currently requires enable_projection_cache=False.")
        if not math.isfinite(capacity_growth_factor) or capacity_growth_factor <= 1.0:
            raise ValueError("capacity_growth_factor must be finite and greater than 1.")
        if not math.isfinite(capacity_headroom) or capacity_headroom < 1.0:
            raise ValueError("capacity_headroom must be finite and at least 1.")
        if (
            isinstance(max_capacity_retries, bool)
            or not isinstance(max_capacity_retries, int)
            or max_capacity_retries < 0
        ):
            raise ValueError("max_capacity_retries must be non-negative.")
        if max_workspace_bytes is not None and max_workspace_bytes <= 0:
            raise ValueError("max_workspace_bytes must be positive when set.")
        if sh_degree is not None and sh_degree not in (0, 1, 2, 3):
            raise ValueError("sh_degree must be None (linear RGB features) or in [0, 3].")
        if tile_size == 2:
            raise ValueError("tile_size=2 is not provided; use 1 (dense mode), 4, 8 or 16.")
        if tile_size == 1 and ray_gaussian_evaluation:
            raise ValueError("dense mode (tile_size=1) renders screen-space evaluation only.")

        self.max_visible_records = max_visible_records
        self.max_intersections = max_intersections
        self.visible_capacity_per_view = visible_capacity_per_view
        self.intersections_per_visible = intersections_per_visible
        self.near_plane = near_plane
        self.far_plane = far_plane
        self.gaussian_support_sigma = gaussian_support_sigma
        self.covariance_epsilon = covariance_epsilon
        self._rasterize_mode: Literal["classic", "antialiased"] = rasterize_mode
        self.semantic_min_alpha = semantic_min_alpha
        self._ray_gaussian_evaluation = bool(ray_gaussian_evaluation)
        self.tile_size = tile_size
        self.depth_bucket_count = depth_bucket_count
        self.depth_bucket_group_size = min(depth_bucket_group_size, depth_bucket_count)
        self.compact_projection_cache = compact_projection_cache
        self.materialize_projected_records = materialize_projected_records
        self.enable_projection_cache = enable_projection_cache
        self.output_srgb = output_srgb
        self.deterministic = deterministic
        self.fixed_capacity_sort = fixed_capacity_sort
        self.max_physical_views = max_physical_views
        self.adaptive_capacity = adaptive_capacity
        self.capacity_growth_factor = capacity_growth_factor
        self.capacity_headroom = capacity_headroom
        self.max_capacity_retries = max_capacity_retries
        self.max_workspace_bytes = max_workspace_bytes
        self.sh_degree = sh_degree
        self.mirror_reference_workspace = mirror_reference_workspace
        # Store registered scenes in Morton order of their means with
        # per-chunk bounds, so that projection skips chunks outside a
        # camera's frustum; every output is unchanged (Gaussians keep their
        # ids).  No counterpart in the reference.
        self.spatial_layout = spatial_layout
        # Compositor as a resident grid over a device work queue (see
        # vgr_render_options.persistent_compositor).
        self.persistent_compositor = persistent_compositor
        # Compositor CTA shape (see vgr_render_options.composite_shape).
        if composite_shape not in (0, 1, 2):
            raise ValueError("composite_shape must be 0, 1 or 2.")
        self.composite_shape = composite_shape
        self._native = native_module
        self._native_loader = native_loader
        self.allow_cpu_for_tests = allow_cpu_for_tests

        self.device: torch.device | None = None
        self.stage: Any | None = None
        self.workspace: dict[str, torch.Tensor] = {}
        self._scenes: OrderedDict[int, GaussianScene] = OrderedDict()
        self._packed_scene: dict[str, torch.Tensor] = {}
        self._max_scene_gaussians = 0
        self._env_scene_ids: torch.Tensor | None = None
        self._env_transforms: torch.Tensor | None = None
        self._max_views = 0
        self._physical_max_views = 0
        self._max_logical_chunks = 1
        self._height = 0
        self._width = 0
        self._scene_revision = 0
        self._workspace_config: tuple[int, int, int, torch.device] | None = None
        self._allocated_visible_capacity = 0
        self._allocated_intersection_capacity = 0
        self._initial_visible_capacity = 0
        self._initial_intersection_capacity = 0
        self._stage_event_handles: Any = None
        self._stage_events_keepalive: list[torch.cuda.Event] = []
        self._reset_stats()

    def _reset_stats(self) -> None:
        self._projection_cache_token: tuple[Any, ...] | None = None
        self._projection_cache_refs: tuple[torch.Tensor, ...] = ()
        self._projection_cache_hits = 0
        self._projection_cache_misses = 0
        self._capacity_validation_token: tuple[Any, ...] | None = None
        self._capacity_validation_refs: tuple[torch.Tensor, ...] = ()
        self._capacity_validation_counters: dict[str, int] | None = None
        self._capacity_validations = 0
        self._capacity_validation_reuses = 0
        self._capacity_growth_events = 0
        self._capacity_total_retries = 0
        self._capacity_last_render: dict[str, Any] | None = None
        self._capacity_last_growth: dict[str, Any] | None = None
        self._capacity_last_allocation: dict[str, Any] | None = None

    # ------------------------------------------------------------------ lifecycle
    def initialize(self, stage: Any, device: torch.device) -> None:
        device = torch.device(device)
        if device.type != "cuda" and not self.allow_cpu_for_tests:
            raise ValueError(f"CustomCudaBackend requires CUDA; got {device}.")
        self.stage = stage
        self.device = device
        if self._native is None:
            self._native = self._native_loader()
        self._reset_stats()

    def register_scene(self, scene_id: int, scene: GaussianScene, offset: int) -> None:
        self._require_initialized()
        expected = sum(registered.count for registered in self._scenes.values())
        if offset != expected:
            raise ValueError(f"Scene {scene_id} offset {offset} does not match packed offset {expected}.")
        width = scene.features.shape[1]
        if width < 3:
            raise ValueError("CustomCudaBackend requires at least three RGB feature channels.")
        if self.sh_degree is not None and width < (self.sh_degree + 1) ** 2 * 3:
            raise ValueError(
                f"sh_degree={self.sh_degree} needs {(self.sh_degree + 1) ** 2 * 3} feature channels; "
                f"got {width}."
            )
        if self._scenes:
            first = next(iter(self._scenes.values())).features.shape[1]
            if width != first:
                raise ValueError(
                    f"All packed scenes must use the same feature width; expected {first}, got {width}."
                )
        self._scenes[scene_id] = scene
        self._rebuild_packed_scene()

    def allocate_workspace(
        self,
        *,
        max_views: int,
        height: int,
        width: int,
        device: torch.device,
        dtype: torch.dtype,
    ) -> dict[str, torch.Tensor]:
        self._require_initialized()
        if dtype != torch.float32:
            raise ValueError("The custom CUDA backend workspace uses float32.")
        if max_views <= 0:
            raise ValueError("max_views must be positive.")
        physical = min(max_views, self.max_physical_views or max_views)
        visible = self.max_visible_records or physical * self.visible_capacity_per_view
        intersections = self.max_intersections or math.ceil(visible * self.intersections_per_visible)
        self._max_views = max_views
        self._physical_max_views = physical
        self._max_logical_chunks = math.ceil(max_views / physical)
        self._height = height
        self._width = width
        self._workspace_config = (physical, height, width, torch.device(device))
        self._install_workspace(visible, intersections, reason="initial-allocation")
        self._initial_visible_capacity = visible
        self._initial_intersection_capacity = intersections
        return self.workspace

    def update_scene_transforms(self, scene_ids: torch.Tensor, transforms: torch.Tensor) -> None:
        self._env_scene_ids = scene_ids
        self._env_transforms = transforms
        self.invalidate_projection_cache()

    def reserve_workspace_capacity(self, *, visible_records: int, tile_intersections: int) -> None:
        """Install an explicit capacity outside measured work."""
        self._require_initialized()
        if not self.workspace:
            raise RuntimeError("allocate_workspace() must be called before reservation.")
        self.synchronize()
        self._install_workspace(
            visible_records, tile_intersections, reason="explicit-benchmark-reservation"
        )

    def synchronize(self) -> None:
        self._require_initialized()
        if self.device is not None and self.device.type == "cuda":
            torch.cuda.synchronize(self.device)

    def shutdown(self) -> None:
        self.invalidate_projection_cache()
        self.workspace = {}
        self._scenes.clear()
        self._packed_scene = {}
        self._env_scene_ids = None
        self._env_transforms = None
        self._workspace_config = None
        self._allocated_visible_capacity = 0
        self._allocated_intersection_capacity = 0
        self.stage = None
        self.device = None

    # --------------------------------------------------------------------- render
    def render(self, request: RenderRequest) -> RenderStats:
        self._require_initialized()
        if not self.workspace:
            raise RuntimeError("allocate_workspace() must be called before render().")
        if not self._packed_scene:
            raise RuntimeError("At least one Gaussian scene must be registered.")
        names = tuple(request.outputs)
        if names not in (RGB_ONLY_OUTPUTS, FULL_SENSOR_OUTPUTS):
            raise ValueError(
                "CustomCudaBackend supports exactly the RGB-only or fused RGB/depth/alpha/semantic_id "
                f"output contract; got {names}."
            )
        full = names == FULL_SENSOR_OUTPUTS
        batch = int(request.camera_transforms.shape[0])
        if batch > self._max_views:
            raise ValueError(f"Render batch {batch} exceeds workspace max_views {self._max_views}.")
        if tuple(request.outputs["rgb"].shape[1:3]) != (self._height, self._width):
            raise ValueError("Output resolution does not match the allocated workspace.")

        attempts: list[dict[str, Any]] = []
        for retry in range(self.max_capacity_retries + 1):
            if batch > self._physical_max_views:
                stats, token, refs = self._submit_chunked(request, full)
            else:
                stats, token, refs = self._submit(request, full)
                if self.max_physical_views is not None:
                    self.workspace["physical_capacity_counters"].copy_(self.workspace["counters"])
            if not self.adaptive_capacity:
                self._capacity_last_render = {
                    "status": "submitted-unvalidated",
                    "validation": "explicit-manual-capacity-mode",
                    "synchronized": False,
                    "retry_count": 0,
                    "attempts": [],
                    "final_capacity": self._capacity_snapshot(),
                    "final_counters": None,
                }
                return stats
            if token is not None and token == self._capacity_validation_token:
                counters = dict(self._capacity_validation_counters or {})
                self._capacity_validation_reuses += 1
                self._capacity_last_render = {
                    "status": "success",
                    "validation": "validated-identical-input",
                    "synchronized": False,
                    "retry_count": retry,
                    "attempts": [self._attempt(retry, counters, "validated-identical-input", False)],
                    "final_capacity": self._capacity_snapshot(),
                    "final_counters": counters,
                }
                return RenderStats(
                    rendered_views=stats.rendered_views,
                    visible_gaussians=counters["visible_gaussians"],
                    tile_intersections=counters["tile_intersections"],
                )
            counters = self.read_counters(synchronize=True)
            self._check_device_status()
            attempt = self._attempt(retry, counters, "device-counters", True)
            attempts.append(attempt)
            if not (counters["visible_overflow"] or counters["intersection_overflow"]):
                self._capacity_validation_token = token
                self._capacity_validation_refs = refs
                self._capacity_validation_counters = dict(counters)
                self._capacity_validations += 1
                self._capacity_total_retries += retry
                record = {
                    "status": "success",
                    "validation": "device-counters",
                    "synchronized": True,
                    "retry_count": retry,
                    "attempts": attempts,
                    "final_capacity": self._capacity_snapshot(),
                    "final_counters": counters,
                }
                self._capacity_last_render = record
                if retry:
                    self._capacity_last_growth = copy.deepcopy(record)
                return RenderStats(
                    rendered_views=stats.rendered_views,
                    visible_gaussians=counters["visible_gaussians"],
                    tile_intersections=counters["tile_intersections"],
                )
            if retry >= self.max_capacity_retries:
                self._capacity_total_retries += retry
                self._raise_capacity_error(
                    request,
                    f"Custom renderer capacity remained insufficient after {retry} bounded retries.",
                    attempts,
                    "retry-limit",
                )
            visible, intersections = self._propose_growth(counters)
            attempt["growth_request"] = {
                "visible_records": visible,
                "tile_intersections": intersections,
            }
            try:
                self._install_workspace(visible, intersections, reason="overflow-retry")
            except RendererCapacityError as error:
                attempt["growth_failure"] = copy.deepcopy(error.telemetry)
                self._capacity_total_retries += retry
                self._raise_capacity_error(
                    request, str(error), attempts, "growth-allocation-failed", cause=error
                )
            self._capacity_growth_events += 1
        raise AssertionError("Unreachable capacity retry state.")

    def _env_for(self, batch: int) -> torch.Tensor:
        if self._env_transforms is None:
            return self.workspace["identity_env_xforms"][:batch]
        if self._env_transforms.shape[0] != batch:
            raise ValueError(
                "update_scene_transforms() must provide one transform per render camera; "
                f"got {self._env_transforms.shape[0]} transforms for batch {batch}."
            )
        return self._env_transforms

    def _reset_inactive(self, outputs: dict[str, torch.Tensor], full: bool) -> None:
        outputs["rgb"].zero_()
        if full:
            outputs["depth"].fill_(float("inf"))
            outputs["alpha"].zero_()
            outputs["semantic_id"].fill_(-1)

    def _submit(
        self, request: RenderRequest, full: bool
    ) -> tuple[RenderStats, tuple[Any, ...] | None, tuple[torch.Tensor, ...]]:
        batch = int(request.camera_transforms.shape[0])
        env = self._env_for(batch)
        active = request.active_camera_ids
        token = self._input_token(batch, request, env, active)
        reuse = self.enable_projection_cache and token == self._projection_cache_token
        if active is not None:
            self._reset_inactive(request.outputs, full)
        self._ensure_scratch(active.numel() if active is not None else batch)
        self._native_render(
            request.camera_transforms,
            request.intrinsics,
            env,
            request.scene_ids,
            active,
            request.outputs,
            full,
            self.workspace["counters"],
            reuse,
        )
        refs = (request.camera_transforms, request.intrinsics, env, request.scene_ids) + (
            (active,) if active is not None else ()
        )
        if self.enable_projection_cache:
            self._projection_cache_token = token
            self._projection_cache_refs = refs
            if reuse:
                self._projection_cache_hits += 1
            else:
                self._projection_cache_misses += 1
        views = int(active.numel()) if active is not None else batch
        return RenderStats(rendered_views=views), token, refs

    def _submit_chunked(
        self, request: RenderRequest, full: bool
    ) -> tuple[RenderStats, tuple[Any, ...] | None, tuple[torch.Tensor, ...]]:
        """One logical request through bounded physical submissions, no host read."""
        batch = int(request.camera_transforms.shape[0])
        physical = self._physical_max_views
        chunks = math.ceil(batch / physical)
        if chunks > self._max_logical_chunks:
            raise ValueError(
                f"Logical batch requires {chunks} chunks but only {self._max_logical_chunks} were allocated."
            )
        env = None if self._env_transforms is None else self._env_for(batch)
        active = request.active_camera_ids
        if active is not None:
            self._reset_inactive(request.outputs, full)
            self._native.prepare_chunked_active_ids(
                active,
                self.workspace["logical_active_mask"],
                self.workspace["logical_chunk_active_ids"],
                batch,
                physical,
            )
        self._ensure_scratch(physical)
        chunk_counters = self.workspace["logical_chunk_counters"]
        for index in range(chunks):
            start = index * physical
            count = min(physical, batch - start)
            sub_outputs = {name: t.narrow(0, start, count) for name, t in request.outputs.items()}
            sub_env = (
                self.workspace["identity_env_xforms"].narrow(0, 0, count)
                if env is None
                else env.narrow(0, start, count)
            )
            sub_active = (
                None
                if active is None
                else self.workspace["logical_chunk_active_ids"][index].narrow(0, 0, count)
            )
            self._native_render(
                request.camera_transforms.narrow(0, start, count),
                request.intrinsics.narrow(0, start, count),
                sub_env,
                request.scene_ids.narrow(0, start, count),
                sub_active,
                sub_outputs,
                full,
                chunk_counters[index],
                False,
            )
        self._native.aggregate_chunk_counters(
            chunk_counters,
            self.workspace["counters"],
            self.workspace["physical_capacity_counters"],
            chunks,
        )
        views = int(active.numel()) if active is not None else batch
        refs = (request.camera_transforms, request.intrinsics, request.scene_ids)
        return RenderStats(rendered_views=views), None, refs

    def _native_render(
        self,
        viewmats: torch.Tensor,
        intrinsics: torch.Tensor,
        env: torch.Tensor,
        scene_ids: torch.Tensor,
        active: torch.Tensor | None,
        outputs: dict[str, torch.Tensor],
        full: bool,
        counters: torch.Tensor,
        reuse: bool,
    ) -> None:
        lib = _native.load_library()
        ws = self.workspace
        packed = self._packed_scene
        scene = self.native_scene()
        # An empty active-id tensor means "every camera", as at the reference's
        # native boundary (renderer_cuda.cu:2626-2628).
        use_active = active is not None and active.numel() > 0
        cams = _native.VgrCameras(
            viewmats=viewmats.data_ptr(),
            intrinsics=intrinsics.data_ptr(),
            env_xforms=env.data_ptr(),
            camera_scene_ids=scene_ids.data_ptr(),
            active_camera_ids=active.data_ptr() if use_active else None,
            batch=viewmats.shape[0],
            active_count=active.numel() if use_active else viewmats.shape[0],
        )
        outs = _native.VgrOutputs(
            rgb=outputs["rgb"].data_ptr(),
            depth=outputs["depth"].data_ptr() if full else None,
            alpha=outputs["alpha"].data_ptr() if full else None,
            semantic=outputs["semantic_id"].data_ptr() if full else None,
        )
        mirror = self.mirror_reference_workspace
        record_rows = self._allocated_visible_capacity * (2 if self._ray_gaussian_evaluation else 1)
        if ws["records"].shape[0] < record_rows:
            # Exact-ray mode switched on after allocation: its extension
            # records follow the records.
            ws["records"] = torch.empty((record_rows, _native.RECORD_BYTES // 4), dtype=torch.float32,
                                        device=self.device)
        native_ws = _native.VgrWorkspace(
            records=ws["records"].data_ptr(),
            visible_capacity=self._allocated_visible_capacity,
            keys_in=ws["keys_in"].data_ptr(),
            keys_out=ws["keys_out"].data_ptr(),
            values_in=ws["values_in"].data_ptr(),
            values_out=ws["values_out"].data_ptr(),
            intersection_capacity=self._allocated_intersection_capacity,
            tile_starts=ws["tile_starts"].data_ptr(),
            tile_ends=ws["tile_ends"].data_ptr(),
            tile_capacity=ws["tile_starts"].numel(),
            counters=counters.data_ptr(),
            scratch=ws["scratch"].data_ptr(),
            scratch_bytes=ws["scratch"].numel(),
            visible_means2d=ws["visible_means2d"].data_ptr() if mirror else None,
            visible_conics=ws["visible_conics"].data_ptr() if mirror else None,
            visible_depths=ws["visible_depths"].data_ptr() if mirror else None,
            visible_opacities=ws["visible_opacities"].data_ptr() if mirror else None,
            visible_camera_ids=ws["visible_camera_ids"].data_ptr() if mirror else None,
            visible_gaussian_ids=ws["visible_gaussian_ids"].data_ptr() if mirror else None,
            visible_radii=ws["visible_radii"].data_ptr() if mirror else None,
            depth_tau=ws["depth_tau"].data_ptr() if self.tile_size == 1 else None,
            depth_tau_capacity=ws["depth_tau"].numel(),
            tile_cutoff=ws["tile_cutoff"].data_ptr() if self.tile_size == 1 else None,
            tile_cutoff_capacity=ws["tile_cutoff"].numel(),
        )
        options = _native.VgrRenderOptions(
            height=self._height,
            width=self._width,
            near_plane=self.near_plane,
            far_plane=self.far_plane,
            gaussian_support_sigma=self.gaussian_support_sigma,
            covariance_epsilon=self.covariance_epsilon,
            semantic_min_alpha=self.semantic_min_alpha,
            antialiased=int(self.rasterize_mode == "antialiased"),
            ray_gaussian_evaluation=int(self._ray_gaussian_evaluation),
            tile_size=self.tile_size,
            output_srgb=int(self.output_srgb),
            deterministic=int(self.deterministic),
            full_sensor_output=int(full),
            fixed_capacity_sort=int(self.fixed_capacity_sort),
            reuse_projection=int(reuse),
            compact_projection_cache=int(self.compact_projection_cache),
            sh_degree=-1 if self.sh_degree is None else self.sh_degree,
            sorted_buffer_hint=1,
            persistent_compositor=int(self.persistent_compositor),
            composite_shape=int(self.composite_shape),
        )
        if self._stage_event_handles is not None:
            options.stage_events = self._stage_event_handles
            options.stage_event_count = _native.STAGE_EVENTS
        selector = _native._c_i64(1)
        assert self.device is not None
        with torch.cuda.device(self.device):
            stream = torch.cuda.current_stream(self.device).cuda_stream
            _native.check(
                lib.vgr_render(scene, cams, outs, native_ws, options, stream, selector), "render"
            )
        if selector.value == 0 and not reuse:
            # Keep values_out/keys_out naming the sorted lists (as the
            # reference backend does after CUB's DoubleBuffer), by swapping
            # the dictionary entries rather than copying.
            ws["keys_in"], ws["keys_out"] = ws["keys_out"], ws["keys_in"]
            ws["values_in"], ws["values_out"] = ws["values_out"], ws["values_in"]

    def native_scene(self) -> _native.VgrScene:
        """The packed scene as the C ABI's vgr_scene (with the spatial
        layout when it is on)."""
        packed = self._packed_scene
        return _native.VgrScene(
            means=packed["means"].data_ptr(),
            covariances=packed["covariances"].data_ptr(),
            opacities=packed["opacities"].data_ptr(),
            features=packed["features"].data_ptr(),
            feature_width=packed["features"].shape[1],
            semantic_ids=packed["semantic_ids"].data_ptr(),
            registered_scene_ids=packed["registered_scene_ids"].data_ptr(),
            scene_offsets=packed["scene_offsets"].data_ptr(),
            scene_count=packed["registered_scene_ids"].numel(),
            gaussian_count=packed["means"].shape[0],
            max_scene_gaussians=self._max_scene_gaussians,
            gaussian_ids=packed["gaussian_ids"].data_ptr() if "gaussian_ids" in packed else None,
            chunk_bounds=packed["chunk_bounds"].data_ptr() if "chunk_bounds" in packed else None,
            chunk_offsets=packed["chunk_offsets"].data_ptr() if "chunk_offsets" in packed else None,
            cluster_bounds=packed["cluster_bounds"].data_ptr() if "cluster_bounds" in packed else None,
        )

    def set_stage_events(self, events: list[torch.cuda.Event] | None) -> None:
        """Record ``events[i]`` at stage boundary i of every native render
        (start, setup, projection, tile scan, bucket scatter, tile sort,
        compositor); None disables.  Used for live per-kernel timing."""
        if events is None:
            self._stage_event_handles = None
            return
        if len(events) != _native.STAGE_EVENTS:
            raise ValueError(f"set_stage_events needs {_native.STAGE_EVENTS} events.")
        stream = torch.cuda.current_stream(self.device)
        for event in events:
            event.record(stream)  # materialise the handle
        self._stage_event_handles = (_native._c_p * _native.STAGE_EVENTS)(
            *[event.cuda_event for event in events]
        )
        self._stage_events_keepalive = list(events)

    # ------------------------------------------------------------------ counters
    def read_counters(self, *, synchronize: bool = True) -> dict[str, int]:
        if synchronize:
            self.synchronize()
        values = self.workspace["counters"].detach().cpu().tolist()
        return dict(zip(COUNTER_NAMES, (int(v) for v in values)))

    def read_physical_capacity_counters(self, *, synchronize: bool = True) -> dict[str, int]:
        if "physical_capacity_counters" not in self.workspace:
            return self.read_counters(synchronize=synchronize)
        if synchronize:
            self.synchronize()
        values = self.workspace["physical_capacity_counters"].detach().cpu().tolist()
        return dict(zip(COUNTER_NAMES, (int(v) for v in values)))

    def read_device_status(self, *, synchronize: bool = True) -> int:
        """Device error bits of the last frame (nonzero: a bounded device wait gave up)."""
        if synchronize:
            self.synchronize()
        return int(self.workspace["scratch"][:4].view(torch.int32).cpu().item())

    def _check_device_status(self) -> None:
        status = self.read_device_status(synchronize=False)
        if status:
            self.invalidate_projection_cache()
            raise RuntimeError(
                f"Renderer device status {status}: a bounded device wait expired; outputs are invalid."
            )

    def check_capacity(self, *, synchronize: bool = True) -> dict[str, int]:
        counters = self.read_counters(synchronize=synchronize)
        if counters["visible_overflow"] or counters["intersection_overflow"]:
            raise RendererCapacityError(
                "Custom renderer workspace overflow: "
                f"visible={counters['visible_overflow']} "
                f"intersections={counters['intersection_overflow']}.",
                telemetry={
                    "schema_version": "renderer-capacity-error/v1",
                    "reason": "explicit-check-overflow",
                    "counters": counters,
                    "capacity": self.capacity_stats,
                },
            )
        return counters

    # ----------------------------------------------------------------- workspace
    def _dense_cells(self) -> int:
        """Optical-thickness cells of dense mode (4x4 pixels) over the batch."""
        assert self._workspace_config is not None
        physical, height, width, _ = self._workspace_config
        cell = _native.DENSE_CELL
        return physical * math.ceil(height / cell) * math.ceil(width / cell)

    def _global_tiles(self) -> int:
        assert self._workspace_config is not None
        physical, height, width, _ = self._workspace_config
        bin_size = self.bin_tile_size
        return physical * math.ceil(height / bin_size) * math.ceil(width / bin_size)

    def _scratch_bytes(self, intersections: int, active: int) -> int:
        lib = _native.load_library()
        return _native.check_size(
            lib.vgr_render_scratch_bytes(
                intersections,
                active * max(self._max_scene_gaussians, 1),
                max(self._global_tiles(), 1),
                active,
            ),
            "render scratch",
        )

    def _ensure_scratch(self, active: int) -> None:
        """Grow the scratch buffer when scenes or the active count outgrow it."""
        need = self._scratch_bytes(self._allocated_intersection_capacity, max(active, 1))
        if self.workspace["scratch"].numel() < need:
            self.workspace["scratch"] = torch.empty(need, dtype=torch.uint8, device=self.device)

    def _workspace_specs(self, visible: int, intersections: int) -> dict[str, tuple[tuple[int, ...], torch.dtype]]:
        assert self._workspace_config is not None
        physical, _, _, _ = self._workspace_config
        if visible > _INT32_MAX:
            raise ValueError("Visible storage capacity exceeds the int32 implementation limit.")
        if intersections > _INT32_MAX:
            raise ValueError("Intersection capacity exceeds the int32 implementation limit.")
        tiles = self._global_tiles()
        specs: dict[str, tuple[tuple[int, ...], torch.dtype]] = {
            # Exact-ray mode stores an extension record after the records.
            "records": ((visible * (2 if self._ray_gaussian_evaluation else 1), _native.RECORD_BYTES // 4),
                        torch.float32),
            "keys_in": ((intersections,), torch.uint64),
            "keys_out": ((intersections,), torch.uint64),
            "values_in": ((intersections,), torch.int32),
            "values_out": ((intersections,), torch.int32),
            # Dense mode: optical-thickness bounds per (tile, depth bucket) and
            # the per-tile depth cutoff.
            "depth_tau": ((self._dense_cells() * _native.DENSE_DEPTH_BUCKETS if self.tile_size == 1 else 1,),
                          torch.float32),
            "tile_cutoff": ((tiles if self.tile_size == 1 else 1,), torch.int32),
            "tile_starts": ((tiles,), torch.int32),
            "tile_ends": ((tiles,), torch.int32),
            "counters": ((len(COUNTER_NAMES),), torch.int64),
            "scratch": ((self._scratch_bytes(intersections, physical),), torch.uint8),
            "identity_env_xforms": ((physical, 4, 4), torch.float32),
            "empty_active_ids": ((0,), torch.int64),
            "dummy_depth": ((1,), torch.float32),
            "dummy_alpha": ((1,), torch.float32),
            "dummy_semantic": ((1,), torch.int64),
        }
        if self.mirror_reference_workspace:
            specs.update(
                {
                    "visible_means2d": ((visible, 2), torch.float32),
                    "visible_conics": ((visible, 3), torch.float32),
                    "visible_depths": ((visible,), torch.float32),
                    "visible_opacities": ((visible,), torch.float32),
                    "visible_camera_ids": ((visible,), torch.int32),
                    "visible_gaussian_ids": ((visible,), torch.int32),
                    "visible_radii": ((visible, 2), torch.int32),
                }
            )
        if self.max_physical_views is not None:
            specs.update(
                {
                    "logical_chunk_counters": ((self._max_logical_chunks, len(COUNTER_NAMES)), torch.int64),
                    "physical_capacity_counters": ((len(COUNTER_NAMES),), torch.int64),
                    "logical_active_mask": ((self._max_views,), torch.int32),
                    "logical_chunk_active_ids": ((self._max_logical_chunks, physical), torch.int64),
                }
            )
        return specs

    @staticmethod
    def _specs_bytes(specs: dict[str, tuple[tuple[int, ...], torch.dtype]]) -> int:
        return sum(
            math.prod(shape) * torch.empty((), dtype=dtype).element_size()
            for shape, dtype in specs.values()
        )

    def _install_workspace(self, visible: int, intersections: int, *, reason: str) -> None:
        try:
            specs = self._workspace_specs(visible, intersections)
        except ValueError as error:
            if reason == "initial-allocation":
                raise
            raise RendererCapacityError(
                str(error),
                telemetry={
                    "schema_version": "renderer-capacity-allocation/v1",
                    "reason": reason,
                    "failure": "native-int32-limit",
                    "requested_capacity": {
                        "visible_records": visible,
                        "tile_intersections": intersections,
                    },
                    "native_limit": _INT32_MAX,
                },
            ) from error
        requested = self._specs_bytes(specs)
        telemetry: dict[str, Any] = {
            "schema_version": "renderer-capacity-allocation/v1",
            "reason": reason,
            "requested_capacity": {"visible_records": visible, "tile_intersections": intersections},
            "requested_workspace_bytes": requested,
            "current_workspace_bytes": self.workspace_bytes,
            "max_workspace_bytes": self.max_workspace_bytes,
        }
        if self.max_workspace_bytes is not None and requested > self.max_workspace_bytes:
            telemetry["failure"] = "workspace-memory-limit"
            telemetry["status"] = "failure"
            self._capacity_last_allocation = copy.deepcopy(telemetry)
            raise RendererCapacityError(
                f"Adaptive capacity growth requires {requested} workspace bytes, exceeding the "
                f"configured limit of {self.max_workspace_bytes} bytes.",
                telemetry=telemetry,
            )
        assert self._workspace_config is not None
        device = self._workspace_config[3]
        release_first = reason in {"overflow-retry", "explicit-benchmark-reservation"} and bool(
            self.workspace
        )
        old = (self._allocated_visible_capacity, self._allocated_intersection_capacity)
        if release_first:
            self.invalidate_projection_cache()
            self.workspace.clear()
            if device.type == "cuda":
                torch.cuda.empty_cache()
        try:
            replacement = {
                name: torch.empty(shape, dtype=dtype, device=device)
                for name, (shape, dtype) in specs.items()
            }
        except torch.OutOfMemoryError as error:
            telemetry["failure"] = "allocator-out-of-memory"
            telemetry["status"] = "failure"
            if release_first:
                try:
                    restored_specs = self._workspace_specs(*old)
                    restored = {
                        name: torch.empty(shape, dtype=dtype, device=device)
                        for name, (shape, dtype) in restored_specs.items()
                    }
                except torch.OutOfMemoryError:
                    self._allocated_visible_capacity = 0
                    self._allocated_intersection_capacity = 0
                    telemetry["restoration"] = {"status": "failed", "workspace_usable": False}
                else:
                    restored["identity_env_xforms"].copy_(
                        torch.eye(4, device=device).repeat(self._workspace_config[0], 1, 1)
                    )
                    self.workspace.update(restored)
                    telemetry["restoration"] = {
                        "status": "restored-old-capacity",
                        "workspace_usable": True,
                        "workspace_bytes": self.workspace_bytes,
                    }
            self._capacity_last_allocation = copy.deepcopy(telemetry)
            raise RendererCapacityError(
                f"CUDA allocator could not satisfy bounded adaptive workspace growth to {requested} bytes.",
                telemetry=telemetry,
            ) from error
        replacement["identity_env_xforms"].copy_(
            torch.eye(4, device=device).repeat(self._workspace_config[0], 1, 1)
        )
        # Keep the dictionary identity that RendererService holds.
        self.workspace.clear()
        self.workspace.update(replacement)
        self._allocated_visible_capacity = visible
        self._allocated_intersection_capacity = intersections
        self.invalidate_projection_cache()
        telemetry["status"] = "success"
        telemetry["installed_workspace_bytes"] = self.workspace_bytes
        self._capacity_last_allocation = copy.deepcopy(telemetry)

    def _propose_growth(self, counters: dict[str, int]) -> tuple[int, int]:
        visible = self._allocated_visible_capacity
        intersections = self._allocated_intersection_capacity
        proposed_visible = visible
        if counters["visible_overflow"]:
            required = max(counters["visible_gaussians"], visible + counters["visible_overflow"])
            proposed_visible = max(
                visible + 1,
                math.ceil(visible * self.capacity_growth_factor),
                math.ceil(required * self.capacity_headroom),
            )
        # The fused emitter counts intersections of every visible record,
        # stored or not, so the demand below is complete even on overflow.
        required_isect = max(
            counters["tile_intersections"], intersections + counters["intersection_overflow"]
        )
        proposed_isect = intersections
        if counters["intersection_overflow"] or proposed_visible > visible:
            proposed_isect = max(
                intersections + 1,
                math.ceil(intersections * self.capacity_growth_factor),
                math.ceil(required_isect * self.capacity_headroom),
            )
        if self.max_workspace_bytes is not None:
            try:
                target = self._specs_bytes(self._workspace_specs(proposed_visible, proposed_isect))
            except ValueError:
                return proposed_visible, proposed_isect
            if target > self.max_workspace_bytes:
                # Relax the headroom down to the observed demand.
                if counters["visible_overflow"]:
                    proposed_visible = max(
                        visible + 1, counters["visible_gaussians"], visible + counters["visible_overflow"]
                    )
                if counters["intersection_overflow"] or proposed_visible > visible:
                    proposed_isect = max(intersections + 1, required_isect)
        return proposed_visible, proposed_isect

    def _capacity_snapshot(self) -> dict[str, int]:
        return {
            "visible_records": self._allocated_visible_capacity,
            "visible_storage_records": self._allocated_visible_capacity,
            "tile_intersections": self._allocated_intersection_capacity,
            "workspace_bytes": self.workspace_bytes,
        }

    def _attempt(self, retry: int, counters: dict[str, int], source: str, synced: bool) -> dict[str, Any]:
        return {
            "attempt": retry + 1,
            "requested_capacity": self._capacity_snapshot(),
            "actual_demand": dict(counters),
            "counter_source": source,
            "synchronized": synced,
            "overflow": bool(counters.get("visible_overflow") or counters.get("intersection_overflow")),
        }

    def _raise_capacity_error(
        self,
        request: RenderRequest,
        message: str,
        attempts: list[dict[str, Any]],
        reason: str,
        cause: BaseException | None = None,
    ) -> NoReturn:
        self.invalidate_projection_cache()
        for name, tensor in request.outputs.items():
            if tensor.is_floating_point():
                tensor.fill_(float("nan"))
            elif name == "semantic_id":
                tensor.fill_(-1)
        self._capacity_last_render = {
            "status": "failure",
            "validation": "device-counters",
            "synchronized": any(a["synchronized"] for a in attempts),
            "retry_count": max(0, len(attempts) - 1),
            "attempts": copy.deepcopy(attempts),
            "final_capacity": self._capacity_snapshot(),
            "final_counters": copy.deepcopy(attempts[-1]["actual_demand"]) if attempts else None,
            "failure_reason": reason,
        }
        if any("growth_request" in a for a in attempts):
            self._capacity_last_growth = copy.deepcopy(self._capacity_last_render)
        if attempts:
            demand = attempts[-1]["actual_demand"]
            requested = attempts[-1]["requested_capacity"]
            message = (
                f"{message} Last attempt: visible_gaussians={demand['visible_gaussians']} "
                f"tile_intersections={demand['tile_intersections']} "
                f"visible_capacity={requested['visible_records']} "
                f"intersection_capacity={requested['tile_intersections']} "
                f"visible_overflow={demand['visible_overflow']} "
                f"intersection_overflow={demand['intersection_overflow']}."
            )
        telemetry = {
            "schema_version": "renderer-capacity-error/v1",
            "reason": reason,
            "capacity": self.capacity_stats,
        }
        if cause is None:
            raise RendererCapacityError(message, telemetry=telemetry)
        raise RendererCapacityError(message, telemetry=telemetry) from cause

    # ------------------------------------------------------------ introspection
    @property
    def workspace_bytes(self) -> int:
        return sum(self.workspace_bytes_by_tensor.values())

    @property
    def workspace_bytes_by_tensor(self) -> dict[str, int]:
        seen: set[tuple[str, int | None, int]] = set()
        result: dict[str, int] = {}
        for name, tensor in self.workspace.items():
            storage = tensor.untyped_storage()
            key = (tensor.device.type, tensor.device.index, int(storage.data_ptr()))
            if storage.nbytes() == 0 or key in seen:
                result[name] = 0
                continue
            seen.add(key)
            result[name] = int(storage.nbytes())
        return result

    @property
    def current_visible_capacity(self) -> int:
        return self._allocated_visible_capacity

    @property
    def current_intersection_capacity(self) -> int:
        return self._allocated_intersection_capacity

    @property
    def visible_storage_capacity(self) -> int:
        return self._allocated_visible_capacity

    @property
    def scene_bytes(self) -> int:
        return sum(t.numel() * t.element_size() for t in self._packed_scene.values())

    @property
    def projection_cache_stats(self) -> dict[str, int | bool]:
        return {
            "enabled": self.enable_projection_cache,
            "hits": self._projection_cache_hits,
            "misses": self._projection_cache_misses,
        }

    @property
    def bin_tile_size(self) -> int:
        """Pixel size of the tiles keys are binned in: dense mode (tile_size 1)
        runs on 16-pixel tiles with its depth cutoff; exact-ray mode bins
        16-pixel tiles as 32 (renderer_cuda.cu:2670-2676)."""
        if self.tile_size == 1:
            return 16
        if self._ray_gaussian_evaluation and self.tile_size == 16:
            return 32
        return self.tile_size

    @property
    def pipeline_name(self) -> str:
        return (
            "b200-ordered-project-emit-device-bounded-onesweep-radix-linear-ranges-"
            "warp-culled-fused-rgba-depth-semantic"
        )

    @property
    def rasterize_mode(self) -> Literal["classic", "antialiased"]:
        return self._rasterize_mode

    @rasterize_mode.setter
    def rasterize_mode(self, value: Literal["classic", "antialiased"]) -> None:
        if value not in ("classic", "antialiased"):
            raise ValueError("rasterize_mode must be 'classic' or 'antialiased'.")
        if value == "antialiased" and self._ray_gaussian_evaluation:
            raise ValueError("rasterize_mode='antialiased' is incompatible with ray_gaussian_evaluation=True.")
        if value != self._rasterize_mode:
            self._rasterize_mode = value
            self.invalidate_projection_cache()

    @property
    def ray_gaussian_evaluation(self) -> bool:
        """Exact ray-Gaussian evaluation (renderer_cuda.cu:795-948,2190-2270)."""
        return self._ray_gaussian_evaluation

    @ray_gaussian_evaluation.setter
    def ray_gaussian_evaluation(self, value: bool) -> None:
        value = bool(value)
        if value and self._rasterize_mode == "antialiased":
            raise ValueError("rasterize_mode='antialiased' is incompatible with ray_gaussian_evaluation=True.")
        if value and self.tile_size == 1:
            raise ValueError("dense mode (tile_size=1) renders screen-space evaluation only.")
        if value != self._ray_gaussian_evaluation:
            tiles_before = self._global_tiles() if self._workspace_config is not None else None
            self._ray_gaussian_evaluation = value
            self.invalidate_projection_cache()
            if tiles_before is not None and self._global_tiles() != tiles_before and self.workspace:
                # The tile grid changed (16-pixel tiles bin as 32 in exact-ray mode).
                self._install_workspace(self._allocated_visible_capacity, self._allocated_intersection_capacity,
                                        reason="ray-mode-switch")

    @property
    def capacity_stats(self) -> dict[str, Any]:
        return {
            "schema_version": "renderer-capacity/v1",
            "policy": "adaptive-bounded-grow-retry" if self.adaptive_capacity else "explicit-manual-check",
            "adaptive": self.adaptive_capacity,
            "initial_capacity": {
                "visible_records": self._initial_visible_capacity,
                "tile_intersections": self._initial_intersection_capacity,
            },
            "current_capacity": self._capacity_snapshot(),
            "execution_schedule": {
                "logical_max_views": self._max_views,
                "physical_max_views": self._physical_max_views,
                "maximum_logical_chunks": self._max_logical_chunks,
                "chunking_enabled": self.max_physical_views is not None,
            },
            "parameters": {
                "rasterize_mode": self.rasterize_mode,
                "covariance_epsilon": self.covariance_epsilon,
                "growth_factor": self.capacity_growth_factor,
                "headroom_factor": self.capacity_headroom,
                "max_retries": self.max_capacity_retries,
                "max_workspace_bytes": self.max_workspace_bytes,
            },
            "totals": {
                "device_validations": self._capacity_validations,
                "validated_input_reuses": self._capacity_validation_reuses,
                "growth_events": self._capacity_growth_events,
                "retries": self._capacity_total_retries,
            },
            "intersection_ordering_synchronization": (
                "device-bounded radix sort: the emitted count never leaves the device"
            ),
            "last_render": copy.deepcopy(self._capacity_last_render),
            "last_growth": copy.deepcopy(self._capacity_last_growth),
            "last_allocation": copy.deepcopy(self._capacity_last_allocation),
        }

    def invalidate_projection_cache(self) -> None:
        """Forget cached geometry and validated capacity (call after writes that
        bypass PyTorch version counters)."""
        self._projection_cache_token = None
        self._projection_cache_refs = ()
        self._capacity_validation_token = None
        self._capacity_validation_refs = ()
        self._capacity_validation_counters = None

    # ----------------------------------------------------------------- helpers
    def _input_token(
        self,
        batch: int,
        request: RenderRequest,
        env: torch.Tensor,
        active: torch.Tensor | None,
    ) -> tuple[Any, ...]:
        packed = self._packed_scene
        return (
            self._scene_revision,
            batch,
            self._height,
            self._width,
            self._max_scene_gaussians,
            self.near_plane,
            self.far_plane,
            self.gaussian_support_sigma,
            self.covariance_epsilon,
            self.rasterize_mode,
            self.tile_size,
            self.sh_degree,
            _tensor_token(packed["means"]),
            _tensor_token(packed["covariances"]),
            _tensor_token(packed["opacities"]),
            _tensor_token(packed["features"]),
            _tensor_token(request.camera_transforms),
            _tensor_token(request.intrinsics),
            _tensor_token(env),
            _tensor_token(request.scene_ids),
            None if active is None else _tensor_token(active),
            self._allocated_visible_capacity,
            self._allocated_intersection_capacity,
        )

    def _spatial_orders(self, scenes: list[GaussianScene]) -> list[torch.Tensor]:
        """Morton order of each scene's means (vgr_scene_spatial_order),
        computed once per registered scene tensor (a registration repacks
        every scene, so the orders of the others are reused)."""
        lib = _native.load_library()
        stream = torch.cuda.current_stream(self.device).cuda_stream
        orders = []
        cache = getattr(self, "_order_cache", {})
        fresh = {}
        for scene in scenes:
            token = (scene.means.data_ptr(), scene.means._version, scene.count)
            cached = cache.get(token)
            if cached is not None:
                orders.append(cached)
                fresh[token] = cached
                continue
            count = scene.count
            temp = torch.empty(
                _native.check_size(lib.vgr_scene_spatial_order_temp_bytes(count), "spatial order"),
                dtype=torch.uint8, device=self.device,
            )
            order = torch.empty(count, dtype=torch.int32, device=self.device)
            means = scene.means.contiguous()
            _native.check(
                lib.vgr_scene_spatial_order(means.data_ptr(), count, order.data_ptr(), temp.data_ptr(),
                                            temp.numel(), stream),
                "spatial order",
            )
            orders.append(order.long())
            fresh[token] = orders[-1]
        self._order_cache = fresh
        return orders

    def _rebuild_packed_scene(self) -> None:
        assert self.device is not None
        scenes = list(self._scenes.values())
        packed: dict[str, torch.Tensor] = {}
        layout = (
            self.spatial_layout
            and self.device.type == "cuda"
            and all(scene.count > 0 for scene in scenes)
        )
        orders = self._spatial_orders(scenes) if layout else None
        for name in ("means", "scales", "rotations", "opacities", "features", "semantic_ids"):
            tensors = [getattr(scene, name) for scene in scenes]
            if orders is not None and name != "semantic_ids":
                # The semantic table stays in id order (it is indexed by id).
                tensors = [t.index_select(0, order) for t, order in zip(tensors, orders)]
            packed[name] = tensors[0] if len(tensors) == 1 else torch.cat(tensors, dim=0).contiguous()
            packed[name] = packed[name].contiguous()
        covariances = torch.empty((packed["scales"].shape[0], 6), device=self.device, dtype=torch.float32)
        self._native.precompute_covariances(packed["scales"], packed["rotations"], covariances)
        packed["covariances"] = covariances
        offsets = [0]
        for scene in scenes:
            offsets.append(offsets[-1] + scene.count)
        if orders is not None:
            lib = _native.load_library()
            stream = torch.cuda.current_stream(self.device).cuda_stream
            packed["gaussian_ids"] = torch.cat(
                [order + off for order, off in zip(orders, offsets[:-1])]
            ).to(torch.int32).contiguous()
            chunk = int(lib.vgr_project_chunk())
            chunk_offsets = [0]
            for scene in scenes:
                chunk_offsets.append(chunk_offsets[-1] + (scene.count + chunk - 1) // chunk)
            bounds = torch.empty((chunk_offsets[-1], 8), dtype=torch.float32, device=self.device)
            clusters_per_chunk = chunk // _native.PROJECT_CLUSTER
            cluster_bounds = torch.empty((chunk_offsets[-1] * clusters_per_chunk, 8), dtype=torch.float32,
                                         device=self.device)
            for s, scene in enumerate(scenes):
                off = offsets[s]
                _native.check(
                    lib.vgr_scene_chunk_bounds(
                        packed["means"][off:].data_ptr(), covariances[off:].data_ptr(), scene.count,
                        bounds[chunk_offsets[s]:].data_ptr(), stream,
                    ),
                    "chunk bounds",
                )
                _native.check(
                    lib.vgr_scene_cluster_bounds(
                        packed["means"][off:].data_ptr(), covariances[off:].data_ptr(), scene.count,
                        cluster_bounds[chunk_offsets[s] * clusters_per_chunk:].data_ptr(), stream,
                    ),
                    "cluster bounds",
                )
            packed["chunk_bounds"] = bounds
            packed["cluster_bounds"] = cluster_bounds
            packed["chunk_offsets"] = torch.tensor(chunk_offsets, device=self.device, dtype=torch.int64)
        packed["registered_scene_ids"] = torch.tensor(list(self._scenes), device=self.device, dtype=torch.int64)
        packed["scene_offsets"] = torch.tensor(offsets, device=self.device, dtype=torch.int64)
        self._packed_scene = packed
        self._max_scene_gaussians = max(scene.count for scene in scenes)
        self._scene_revision += 1
        self.invalidate_projection_cache()
        if self.workspace:
            physical = self._physical_max_views
            self._ensure_scratch(physical)

    def _require_initialized(self) -> None:
        if self.device is None:
            raise RuntimeError("CustomCudaBackend.initialize() must be called first.")
