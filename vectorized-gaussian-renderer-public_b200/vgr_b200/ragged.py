"""Ragged batched submission: cameras of different resolutions, each looking
at any registered scene, rendered as one logical submission.

The plain form (``RendererService`` / ``CustomCudaBackend.render``, the
reference's drop-in) renders B cameras of one resolution per call, so a rig
of mixed resolutions over several scenes takes one call per (resolution)
group.  ``RaggedBatch`` takes the whole rig at once:

* per-camera tile and pixel offsets are computed once on the host from the
  resolution list (no device round trip) and uploaded once;
* outputs are flat pixel-major buffers (``rgb [P,3]``, ``depth``/``alpha``
  ``[P,1]``, ``semantic_id [P,1]``) with per-camera views;
* the workspace is sized by one calibration render whose counters are read
  back; steady-state frames then run with no host synchronisation, so a frame
  (or a sequence of them) can be captured in a CUDA graph and replayed with
  new poses written into the same input tensors;
* the tile size is chosen per shape class by a small autotuner
  (``autotune_tile_size``) that times the candidates on the actual rig.

The scene data, projection options and SH degree come from a
``CustomCudaBackend`` whose scenes are registered (its own workspace is not
used).  Kernels, parity and the arithmetic contract are those of the plain
form: the ragged form is the same C-ABI entry point (``vgr_render``) with the
per-camera ``widths``/``heights``/``tile_offsets``/``pixel_offsets`` set.
"""

from __future__ import annotations

import math
from collections.abc import Sequence
from typing import Any

import torch

from . import _native
from .cuda_backend import COUNTER_NAMES, CustomCudaBackend, RendererCapacityError

OUTPUT_NAMES = ("rgb", "depth", "alpha", "semantic_id")


class RaggedBatch:
    def __init__(
        self,
        backend: CustomCudaBackend,
        heights: Sequence[int],
        widths: Sequence[int],
        *,
        tile_size: int | None = None,
        full_sensor_output: bool = True,
        headroom: float = 1.25,
        persistent_compositor: bool = False,
        composite_shape: int = 2,
    ) -> None:
        if backend.device is None or not backend._packed_scene:
            raise RuntimeError("RaggedBatch needs an initialized backend with registered scenes.")
        if len(heights) != len(widths) or not heights:
            raise ValueError("heights and widths must be non-empty and of equal length.")
        if any(int(h) <= 0 or int(w) <= 0 for h, w in zip(heights, widths)):
            raise ValueError("every camera needs a positive resolution.")
        self.backend = backend
        self.device = backend.device
        self.heights = [int(h) for h in heights]
        self.widths = [int(w) for w in widths]
        self.batch = len(self.heights)
        self.full = bool(full_sensor_output)
        self.headroom = float(headroom)
        # Compositor as a resident grid over the device work queue of
        # (camera, tile) items instead of one CTA per item slot (the grid of
        # a ragged batch is sized for its largest camera).  Off by default:
        # on the 1,024-camera frame both take 11.0 ms (the empty slots exit at
        # once and the hardware scheduler balances the rest).
        self.persistent_compositor = bool(persistent_compositor)
        # Compositor CTA shape (vgr_render_options.composite_shape): 0 two
        # pixels per thread, 1 one pixel per thread, 2 (the default) two
        # pixels per thread at half occupancy with 512-record batches; every
        # shape renders the same bits.
        self.composite_shape = int(composite_shape)
        self.tile_size = int(tile_size or backend.tile_size)
        self._visible_capacity = 0
        self._intersection_capacity = 0
        self._stage_events = None
        self.autotune_ms: dict[int, float] = {}
        self.workspace: dict[str, torch.Tensor] = {}
        pixel_offsets = [0]
        for h, w in zip(self.heights, self.widths):
            pixel_offsets.append(pixel_offsets[-1] + h * w)
        self.pixel_offsets_host = pixel_offsets
        self.total_pixels = pixel_offsets[-1]
        dev = self.device
        self._heights_t = torch.tensor(self.heights, dtype=torch.int32, device=dev)
        self._widths_t = torch.tensor(self.widths, dtype=torch.int32, device=dev)
        self._pixel_offsets_t = torch.tensor(pixel_offsets, dtype=torch.int64, device=dev)
        self._env = torch.eye(4, device=dev, dtype=torch.float32).repeat(self.batch, 1, 1).contiguous()
        self._set_tiles(self.tile_size)

    # ------------------------------------------------------------ layout
    def _set_tiles(self, tile_size: int) -> None:
        if tile_size not in (4, 8, 16, 32):
            raise ValueError("tile_size must be 4, 8, 16 or 32.")
        self.tile_size = tile_size
        offsets = [0]
        most = 0
        for h, w in zip(self.heights, self.widths):
            tiles = math.ceil(h / tile_size) * math.ceil(w / tile_size)
            offsets.append(offsets[-1] + tiles)
            most = max(most, tiles)
        self.total_tiles = offsets[-1]
        self.max_tiles_per_camera = most
        self._tile_offsets_t = torch.tensor(offsets, dtype=torch.int64, device=self.device)
        if self.workspace:
            self._install(self._visible_capacity, self._intersection_capacity)

    def outputs(self) -> dict[str, torch.Tensor]:
        """Flat output buffers for the whole rig."""
        dev, p = self.device, self.total_pixels
        out = {"rgb": torch.zeros((p, 3), device=dev, dtype=torch.float32)}
        if self.full:
            out["depth"] = torch.full((p, 1), float("inf"), device=dev, dtype=torch.float32)
            out["alpha"] = torch.zeros((p, 1), device=dev, dtype=torch.float32)
            out["semantic_id"] = torch.full((p, 1), -1, device=dev, dtype=torch.int64)
        return out

    def view(self, outputs: dict[str, torch.Tensor], name: str, camera: int) -> torch.Tensor:
        """Camera ``camera``'s image of output ``name`` as ``[H, W, C]``."""
        a, b = self.pixel_offsets_host[camera], self.pixel_offsets_host[camera + 1]
        return outputs[name][a:b].view(self.heights[camera], self.widths[camera], -1)

    # --------------------------------------------------------- workspace
    def _install(self, visible: int, intersections: int) -> None:
        dev = self.device
        lib = _native.load_library()
        scratch = _native.check_size(
            lib.vgr_render_scratch_bytes(
                intersections,
                self.batch * max(self.backend._max_scene_gaussians, 1),
                max(self.total_tiles, 1),
                self.batch,
            ),
            "ragged render scratch",
        )
        self.workspace = {
            "records": torch.empty((self._record_rows(visible), 12), device=dev, dtype=torch.float32),
            "keys_in": torch.empty((intersections,), device=dev, dtype=torch.uint64),
            "keys_out": torch.empty((intersections,), device=dev, dtype=torch.uint64),
            "values_in": torch.empty((intersections,), device=dev, dtype=torch.int32),
            "values_out": torch.empty((intersections,), device=dev, dtype=torch.int32),
            "tile_starts": torch.empty((self.total_tiles,), device=dev, dtype=torch.int32),
            "tile_ends": torch.empty((self.total_tiles,), device=dev, dtype=torch.int32),
            "counters": torch.zeros((5,), device=dev, dtype=torch.int64),
            "scratch": torch.empty((scratch,), device=dev, dtype=torch.uint8),
        }
        self._visible_capacity = visible
        self._intersection_capacity = intersections

    def _record_rows(self, visible: int) -> int:
        # Exact-ray mode stores an extension record after the records.
        return visible * (2 if self.backend.ray_gaussian_evaluation else 1)

    def reserve(self, *, visible_records: int, tile_intersections: int) -> None:
        """Allocate the workspace for at least these counts (no render)."""
        self._install(max(int(visible_records), 1), max(int(tile_intersections), 1))

    @property
    def capacity(self) -> tuple[int, int]:
        return self._visible_capacity, self._intersection_capacity

    def workspace_bytes(self) -> int:
        return sum(t.numel() * t.element_size() for t in self.workspace.values())

    # ------------------------------------------------------------ render
    def render(
        self,
        viewmats: torch.Tensor,
        intrinsics: torch.Tensor,
        scene_ids: torch.Tensor,
        outputs: dict[str, torch.Tensor],
    ) -> None:
        """Enqueue one frame on the current stream (no host synchronisation)."""
        if not self.workspace:
            raise RuntimeError("call calibrate() or reserve() before render().")
        if viewmats.shape != (self.batch, 4, 4) or intrinsics.shape != (self.batch, 3, 3):
            raise ValueError("viewmats [B,4,4] and intrinsics [B,3,3] must match the rig.")
        if scene_ids.shape != (self.batch,) or scene_ids.dtype != torch.int64:
            raise ValueError("scene_ids must be int64 [B].")
        for t in (viewmats, intrinsics, scene_ids):
            if t.device != self.device or not t.is_contiguous():
                raise ValueError("ragged inputs must be contiguous tensors on the backend's device.")
        if outputs["rgb"].shape != (self.total_pixels, 3):
            raise ValueError("outputs must come from RaggedBatch.outputs().")
        b = self.backend
        lib = _native.load_library()
        ws = self.workspace
        if ws["records"].shape[0] < self._record_rows(self._visible_capacity):
            ws["records"] = torch.empty((self._record_rows(self._visible_capacity), 12), device=self.device,
                                        dtype=torch.float32)
        scene = b.native_scene()
        cams = _native.VgrCameras(
            viewmats=viewmats.data_ptr(),
            intrinsics=intrinsics.data_ptr(),
            env_xforms=self._env.data_ptr(),
            camera_scene_ids=scene_ids.data_ptr(),
            active_camera_ids=None,
            batch=self.batch,
            active_count=self.batch,
            widths=self._widths_t.data_ptr(),
            heights=self._heights_t.data_ptr(),
            tile_offsets=self._tile_offsets_t.data_ptr(),
            pixel_offsets=self._pixel_offsets_t.data_ptr(),
            total_tiles=self.total_tiles,
            max_tiles_per_camera=self.max_tiles_per_camera,
        )
        outs = _native.VgrOutputs(
            rgb=outputs["rgb"].data_ptr(),
            depth=outputs["depth"].data_ptr() if self.full else None,
            alpha=outputs["alpha"].data_ptr() if self.full else None,
            semantic=outputs["semantic_id"].data_ptr() if self.full else None,
        )
        native_ws = _native.VgrWorkspace(
            records=ws["records"].data_ptr(),
            visible_capacity=self._visible_capacity,
            keys_in=ws["keys_in"].data_ptr(),
            keys_out=ws["keys_out"].data_ptr(),
            values_in=ws["values_in"].data_ptr(),
            values_out=ws["values_out"].data_ptr(),
            intersection_capacity=self._intersection_capacity,
            tile_starts=ws["tile_starts"].data_ptr(),
            tile_ends=ws["tile_ends"].data_ptr(),
            tile_capacity=self.total_tiles,
            counters=ws["counters"].data_ptr(),
            scratch=ws["scratch"].data_ptr(),
            scratch_bytes=ws["scratch"].numel(),
        )
        options = _native.VgrRenderOptions(
            height=max(self.heights),
            width=max(self.widths),
            near_plane=b.near_plane,
            far_plane=b.far_plane,
            gaussian_support_sigma=b.gaussian_support_sigma,
            covariance_epsilon=b.covariance_epsilon,
            semantic_min_alpha=b.semantic_min_alpha,
            antialiased=int(b.rasterize_mode == "antialiased"),
            ray_gaussian_evaluation=int(b.ray_gaussian_evaluation),
            tile_size=self.tile_size,
            output_srgb=int(b.output_srgb),
            deterministic=int(b.deterministic),
            full_sensor_output=int(self.full),
            sh_degree=-1 if b.sh_degree is None else b.sh_degree,
            sorted_buffer_hint=1,
            persistent_compositor=int(self.persistent_compositor),
            composite_shape=self.composite_shape,
        )
        if self._stage_events is not None:
            options.stage_events = self._stage_events
            options.stage_event_count = _native.STAGE_EVENTS
        selector = _native._c_i64(1)
        stream = torch.cuda.current_stream(self.device).cuda_stream
        _native.check(lib.vgr_render(scene, cams, outs, native_ws, options, stream, selector), "ragged render")

    def set_stage_events(self, events: list[torch.cuda.Event] | None) -> None:
        """Record ``events[i]`` at the native stage boundaries of every render
        (as ``CustomCudaBackend.set_stage_events``); None disables."""
        if events is None:
            self._stage_events = None
            return
        if len(events) != _native.STAGE_EVENTS:
            raise ValueError(f"need {_native.STAGE_EVENTS} events")
        stream = torch.cuda.current_stream(self.device)
        for event in events:
            event.record(stream)  # materialise the handle
        handles = (_native._c_p * len(events))(*[event.cuda_event for event in events])
        self._events_keepalive = list(events)
        self._stage_events = handles

    def read_counters(self) -> dict[str, int]:
        values = self.workspace["counters"].detach().cpu().tolist()
        return dict(zip(COUNTER_NAMES, (int(v) for v in values)))

    def check(self) -> dict[str, int]:
        """Synchronise and raise RendererCapacityError if the last frame overflowed."""
        counters = self.read_counters()
        if counters["visible_overflow"] or counters["intersection_overflow"]:
            raise RendererCapacityError(
                "ragged batch capacity exceeded; call calibrate() again",
                telemetry={"counters": counters, "capacity": self.capacity},
            )
        return counters

    def calibrate(
        self,
        viewmats: torch.Tensor,
        intrinsics: torch.Tensor,
        scene_ids: torch.Tensor,
        outputs: dict[str, torch.Tensor],
        *,
        max_rounds: int = 4,
    ) -> dict[str, int]:
        """Render, read the counters and grow until the frame fits, leaving
        ``headroom`` for pose changes.  The only synchronising call."""
        if not self.workspace:
            self._install(1 << 16, 1 << 18)
        for _ in range(max_rounds):
            self.render(viewmats, intrinsics, scene_ids, outputs)
            counters = self.read_counters()
            visible, isects = counters["visible_gaussians"], counters["tile_intersections"]
            fits = visible <= self._visible_capacity and isects <= self._intersection_capacity
            want_v = math.ceil(visible * self.headroom) + 1
            want_i = math.ceil(isects * self.headroom) + 1
            if fits and want_v <= self._visible_capacity and want_i <= self._intersection_capacity:
                return counters
            self._install(max(want_v, self._visible_capacity), max(want_i, self._intersection_capacity))
        self.render(viewmats, intrinsics, scene_ids, outputs)
        return self.check()

    def capture(
        self,
        viewmats: torch.Tensor,
        intrinsics: torch.Tensor,
        scene_ids: torch.Tensor,
        outputs: dict[str, torch.Tensor],
        frames: int = 1,
    ) -> torch.cuda.CUDAGraph:
        """Capture ``frames`` renders of the current inputs into a CUDA graph;
        replay after writing new poses into ``viewmats``/``intrinsics``."""
        graph = torch.cuda.CUDAGraph()
        side = torch.cuda.Stream(self.device)
        side.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.stream(side):
            self.render(viewmats, intrinsics, scene_ids, outputs)  # warm the capture stream
        torch.cuda.current_stream(self.device).wait_stream(side)
        torch.cuda.synchronize(self.device)
        with torch.cuda.graph(graph):
            for _ in range(frames):
                self.render(viewmats, intrinsics, scene_ids, outputs)
        return graph


def autotune_tile_size(
    ragged: RaggedBatch,
    viewmats: torch.Tensor,
    intrinsics: torch.Tensor,
    scene_ids: torch.Tensor,
    outputs: dict[str, torch.Tensor],
    *,
    candidates: Sequence[int] = (8, 16, 32),
    persistent_candidates: Sequence[bool] = (False,),
    shape_candidates: Sequence[int] = (0,),
    repeats: int = 3,
    cache: dict[Any, Any] | None = None,
) -> int:
    """Pick the fastest tile size and compositor launch for this rig's shape
    class: tile size x (with ``persistent_candidates``) one CTA per tile or
    the resident work-queue grid x (with ``shape_candidates``) the
    compositor's CTA shape (composite_shape: pixels per thread and
    occupancy; 4-pixel tiles have one shape, and on 8-pixel tiles shapes 0
    and 2 coincide).  Each candidate is timed on the device after
    calibrating its workspace; ``ragged`` is left set to the winner.
    ``cache`` maps shape classes (resolution multiset, camera count, scene
    sizes) to earlier choices.  Returns the tile size; the launch choices are
    on ``ragged`` (``persistent_compositor``, ``composite_shape``) and every
    timing in ``ragged.autotune_ms``."""
    key = (
        tuple(sorted(set(zip(ragged.heights, ragged.widths)))),
        ragged.batch,
        tuple(s.count for s in ragged.backend._scenes.values()),
        tuple(candidates),
        tuple(persistent_candidates),
        tuple(shape_candidates),
    )

    def apply(choice) -> None:
        tile, persistent, shape = choice
        ragged.persistent_compositor = persistent
        ragged.composite_shape = shape
        ragged._set_tiles(tile)
        ragged.calibrate(viewmats, intrinsics, scene_ids, outputs)

    if cache is not None and key in cache:
        apply(cache[key])
        return cache[key][0]
    best, best_ms = None, float("inf")
    stream = torch.cuda.current_stream(ragged.device)
    for persistent in persistent_candidates:
        for tile in candidates:
            for shape in shape_candidates:
                if (tile == 4 and shape != 0) or (tile == 8 and shape == 2):
                    continue  # the same kernel as shape 0
                apply((tile, persistent, shape))
                start = torch.cuda.Event(enable_timing=True)
                stop = torch.cuda.Event(enable_timing=True)
                start.record(stream)
                for _ in range(repeats):
                    ragged.render(viewmats, intrinsics, scene_ids, outputs)
                stop.record(stream)
                stop.synchronize()
                ms = start.elapsed_time(stop) / repeats
                label = str(tile)
                if len(persistent_candidates) > 1 and persistent:
                    label += "p"
                if len(shape_candidates) > 1:
                    label += f"s{shape}"
                ragged.autotune_ms[label if label != str(tile) else tile] = ms
                if ms < best_ms:
                    best, best_ms = (tile, persistent, shape), ms
    assert best is not None
    apply(best)
    if cache is not None:
        cache[key] = best
    return best[0]
