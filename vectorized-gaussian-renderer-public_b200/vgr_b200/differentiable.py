"""Differentiable form of the camera path: ``torch.autograd`` over the native
training forward and hand-written backward kernels.

The reference renders forward only (``renderer_cuda.cu:1973-2305`` over the
projection of ``:287-490``) and measures gradients through gsplat's
``rasterization`` (``benchmarks/compare_custom_gsplat.py:1163-1203``).  This
module trains the same image-formation equation: parameters are the raw
optimisation variables (means, log scales, WXYZ quaternions of any norm,
opacity logits, SH coefficients), the forward applies ``exp``, ``q / |q|`` and
``sigmoid`` in ``vgr_train_activate`` and renders RGB, depth and alpha with
``vgr_render_train``; the backward (``vgr_render_backward``) runs the
compositor backward and one pass per Gaussian through the projection, the SH
colour model and the activations.  All of it runs on the caller's current CUDA
stream; there is no CPU fallback.

One frame is in flight per renderer: the backward reads the forward's sorted
lists and per-pixel state from the renderer's workspace, so call
``backward`` (or let autograd do it) before the next ``render``.

Memory budget (``list_budget_bytes``): the lists a frame keeps for its
backward (24 B per tile intersection, 96 B per visible record, 4 B per
(camera, Gaussian) record-map entry) grow with the batch.  When a batch's
lists would exceed the budget, the forward renders the cameras in chunks
whose lists fit, keeping only the per-pixel state (final transmittance and
last blended position, 8 B per pixel), and the backward recomputes each
chunk's lists (projection, emission, sort) before its backward kernels,
summing the chunks' parameter gradients.
"""

from __future__ import annotations

import math
from typing import Any

import torch

from . import _native

_INT32_MAX = 2**31 - 1


class DifferentiableRenderer:
    """Batched differentiable renderer of one scene seen by ``B`` cameras.

    ``render`` returns ``(rgb [B,H,W,3], depth [B,H,W,1], alpha [B,H,W,1])``;
    depth is ``+inf`` where alpha <= 1e-8, as in the forward contract.
    """

    def __init__(
        self,
        *,
        height: int,
        width: int,
        sh_degree: int = 3,
        tile_size: int = 16,
        near_plane: float = 0.01,
        far_plane: float = 100.0,
        gaussian_support_sigma: float = 3.33,
        covariance_epsilon: float = 0.3,
        headroom: float = 1.25,
        capacity_check: str = "sync",
        device: torch.device | str | None = None,
        list_budget_bytes: int | None = None,
    ) -> None:
        if height <= 0 or width <= 0:
            raise ValueError("height and width must be positive")
        if sh_degree not in (-1, 0, 1, 2, 3):
            raise ValueError("sh_degree must be -1 (linear RGB features) or in [0, 3]")
        if tile_size not in (4, 8, 16):
            raise ValueError("tile_size must be 4, 8 or 16")
        if capacity_check not in ("sync", "deferred"):
            raise ValueError("capacity_check must be 'sync' or 'deferred'")
        if list_budget_bytes is not None and list_budget_bytes <= 0:
            raise ValueError("list_budget_bytes must be positive when set")
        self.list_budget_bytes = list_budget_bytes
        self._bytes_per_camera: float | None = None
        self._calibrated_cameras = 0
        self.capacity_check = capacity_check
        self.height = int(height)
        self.width = int(width)
        self.sh_degree = int(sh_degree)
        self.tile_size = int(tile_size)
        self.near_plane = float(near_plane)
        self.far_plane = float(far_plane)
        self.gaussian_support_sigma = float(gaussian_support_sigma)
        self.covariance_epsilon = float(covariance_epsilon)
        self.headroom = float(headroom)
        self.device = torch.device(device) if device is not None else None
        if self.device is not None and self.device.type == "cuda" and self.device.index is None:
            self.device = torch.device("cuda", torch.cuda.current_device())
        self._lib = _native.load_library()
        self._ws: dict[str, torch.Tensor] = {}
        self._visible_capacity = 0
        self._intersection_capacity = 0
        self._frame = 0
        self._pending: dict[str, Any] | None = None
        self._key: tuple[Any, ...] | None = None
        self._calibrated = False
        self._host_counters: torch.Tensor | None = None
        self.last_counters: dict[str, int] = {}

    # ------------------------------------------------------------------ API
    def render(
        self,
        means: torch.Tensor,
        log_scales: torch.Tensor,
        rotations: torch.Tensor,
        opacity_logits: torch.Tensor,
        features: torch.Tensor,
        viewmats: torch.Tensor,
        intrinsics: torch.Tensor,
    ) -> tuple[torch.Tensor, torch.Tensor, torch.Tensor]:
        return _RenderFunction.apply(
            self, means, log_scales, rotations, opacity_logits, features, viewmats, intrinsics
        )

    # --------------------------------------------------------------- forward
    def _check_inputs(self, means, log_scales, rotations, opacity_logits, features, viewmats, intrinsics):
        device = means.device
        if device.type != "cuda":
            raise ValueError("the differentiable renderer runs on CUDA tensors only")
        if self.device is not None and device != self.device:
            raise ValueError(f"inputs are on {device}, the renderer on {self.device}")
        g = means.shape[0]
        expect = {
            "means": (means, (g, 3)),
            "log_scales": (log_scales, (g, 3)),
            "rotations": (rotations, (g, 4)),
            "opacity_logits": (opacity_logits, (g,)),
        }
        for name, (tensor, shape) in expect.items():
            if tuple(tensor.shape) != shape:
                raise ValueError(f"{name} must have shape {list(shape)}, got {list(tensor.shape)}")
        need = 3 if self.sh_degree < 0 else (self.sh_degree + 1) ** 2 * 3
        if features.dim() != 2 or features.shape[0] != g or features.shape[1] < need:
            raise ValueError(f"features must have shape [G, >={need}]")
        b = viewmats.shape[0]
        if tuple(viewmats.shape) != (b, 4, 4) or tuple(intrinsics.shape) != (b, 3, 3):
            raise ValueError("viewmats must be [B,4,4] and intrinsics [B,3,3]")
        for t in (means, log_scales, rotations, opacity_logits, features, viewmats, intrinsics):
            if t.dtype != torch.float32:
                raise ValueError("all inputs must be float32")
            if t.device != device:
                raise ValueError("all inputs must be on one device")
        if g == 0 or g > _INT32_MAX:
            raise ValueError("the scene must hold between 1 and 2^31-1 Gaussians")

    def _ensure(self, name: str, shape: tuple[int, ...], dtype: torch.dtype, device) -> torch.Tensor:
        t = self._ws.get(name)
        if t is None or t.dtype != dtype or t.device != device or t.numel() < math.prod(shape):
            t = torch.empty(shape, dtype=dtype, device=device)
            self._ws[name] = t
        return t

    def _prepare(self, g: int, b: int, device) -> None:
        ts = self.tile_size
        tiles = b * math.ceil(self.height / ts) * math.ceil(self.width / ts)
        pixels = b * self.height * self.width
        if self._visible_capacity == 0:
            # Every (camera, Gaussian) pair can be visible at most once (with a
            # list budget the first render is one camera; capacity grows).
            cams = 1 if self.list_budget_bytes is not None else b
            self._visible_capacity = min(cams * g, _INT32_MAX)
            self._intersection_capacity = min(max(4 * cams * g, 1024), _INT32_MAX)
        key = (g, b, device)
        if self._key == key:
            return
        self._key = key
        self._ensure("covariances", (g, 6), torch.float32, device)
        self._ensure("opacities", (g,), torch.float32, device)
        self._ensure("semantic_ids", (g,), torch.int64, device).zero_()
        self._ws["registered_scene_ids"] = torch.zeros(1, dtype=torch.int64, device=device)
        self._ws["scene_offsets"] = torch.tensor([0, g], dtype=torch.int64, device=device)
        self._ws["camera_scene_ids"] = torch.zeros(b, dtype=torch.int64, device=device)
        self._ws["env_xforms"] = torch.eye(4, device=device).expand(b, 4, 4).contiguous()
        self._ensure("tile_starts", (tiles,), torch.int32, device)
        self._ensure("tile_ends", (tiles,), torch.int32, device)
        self._ensure("counters", (5,), torch.int64, device)
        self._ensure("final_transmittance", (pixels,), torch.float32, device)
        self._ensure("last_position", (pixels,), torch.int32, device)
        self._ensure("record_map", (b * g,), torch.int32, device)
        self._ensure("semantic_out", (pixels,), torch.int64, device)
        scratch = _native.check_size(self._lib.vgr_render_scratch_bytes(1, b * g, tiles, b), "render scratch")
        self._ensure("scratch", (scratch,), torch.uint8, device)
        self._grow(device)

    def _grow(self, device) -> None:
        v, i = self._visible_capacity, self._intersection_capacity
        self._ensure("records", (v, _native.RECORD_BYTES // 4), torch.float32, device)
        self._ensure("record_grads", (v, _native.RECORD_BYTES // 4), torch.float32, device)
        for name in ("keys_in", "keys_out"):
            self._ensure(name, (i,), torch.uint64, device)
        for name in ("values_in", "values_out"):
            self._ensure(name, (i,), torch.int32, device)

    def _structs(self, means, features, viewmats, intrinsics, rgb, depth, alpha, cam0: int = 0):
        ws = self._ws
        g = means.shape[0]
        b = viewmats.shape[0]
        scene = _native.VgrScene(
            means=means.data_ptr(),
            covariances=ws["covariances"].data_ptr(),
            opacities=ws["opacities"].data_ptr(),
            features=features.data_ptr(),
            feature_width=features.shape[1],
            semantic_ids=ws["semantic_ids"].data_ptr(),
            registered_scene_ids=ws["registered_scene_ids"].data_ptr(),
            scene_offsets=ws["scene_offsets"].data_ptr(),
            scene_count=1,
            gaussian_count=g,
            max_scene_gaussians=g,
        )
        cams = _native.VgrCameras(
            viewmats=viewmats.data_ptr(),
            intrinsics=intrinsics.data_ptr(),
            env_xforms=ws["env_xforms"].data_ptr(),
            camera_scene_ids=ws["camera_scene_ids"].data_ptr(),
            active_camera_ids=None,
            batch=b,
            active_count=b,
        )
        outs = _native.VgrOutputs(
            rgb=rgb.data_ptr(), depth=depth.data_ptr(), alpha=alpha.data_ptr(),
            semantic=ws["semantic_out"].data_ptr(),
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
            tile_capacity=ws["tile_starts"].numel(),
            counters=ws["counters"].data_ptr(),
            scratch=ws["scratch"].data_ptr(),
            scratch_bytes=ws["scratch"].numel(),
        )
        options = _native.VgrRenderOptions(
            height=self.height,
            width=self.width,
            near_plane=self.near_plane,
            far_plane=self.far_plane,
            gaussian_support_sigma=self.gaussian_support_sigma,
            covariance_epsilon=self.covariance_epsilon,
            semantic_min_alpha=0.01,
            antialiased=0,
            ray_gaussian_evaluation=0,
            tile_size=self.tile_size,
            output_srgb=0,
            deterministic=1,
            full_sensor_output=1,
            fixed_capacity_sort=1,
            reuse_projection=0,
            compact_projection_cache=0,
            sh_degree=self.sh_degree,
            sorted_buffer_hint=1,
        )
        px0 = cam0 * self.height * self.width  # per-pixel state of this camera range
        state = _native.VgrTrainState(
            final_transmittance=ws["final_transmittance"][px0:].data_ptr(),
            last_position=ws["last_position"][px0:].data_ptr(),
            record_map=ws["record_map"].data_ptr(),
            record_map_capacity=ws["record_map"].numel(),
            record_grads=ws["record_grads"].data_ptr(),
        )
        return scene, cams, outs, native_ws, options, state

    def forward_native(self, means, log_scales, rotations, opacity_logits, features, viewmats, intrinsics):
        """Training forward without autograd bookkeeping; returns the outputs."""
        self._check_inputs(means, log_scales, rotations, opacity_logits, features, viewmats, intrinsics)
        means, log_scales, rotations, opacity_logits, features, viewmats, intrinsics = (
            t.contiguous() for t in (means, log_scales, rotations, opacity_logits, features, viewmats, intrinsics)
        )
        device = means.device
        g, b = means.shape[0], viewmats.shape[0]
        self._prepare(g, b, device)
        stream = torch.cuda.current_stream(device).cuda_stream
        params = _native.VgrTrainParams(
            log_scales=log_scales.data_ptr(), rotations=rotations.data_ptr(),
            opacity_logits=opacity_logits.data_ptr(),
        )
        _native.check(
            self._lib.vgr_train_activate(params, g, self._ws["covariances"].data_ptr(),
                                         self._ws["opacities"].data_ptr(), stream),
            "train_activate",
        )
        rgb = torch.empty((b, self.height, self.width, 3), dtype=torch.float32, device=device)
        depth = torch.empty((b, self.height, self.width, 1), dtype=torch.float32, device=device)
        alpha = torch.empty((b, self.height, self.width, 1), dtype=torch.float32, device=device)
        tensors = (means, log_scales, rotations, opacity_logits, features, viewmats, intrinsics)
        chunks = self._camera_chunks(b)
        self._reserve_host_counters(len(chunks))
        counter_event = None
        for slot, (s, e) in enumerate(chunks):
            event = self._render_range(tensors, (rgb, depth, alpha), s, e, allow_deferred=True, slot=slot)
            counter_event = event or counter_event
        self._frame += 1
        self._pending = {
            "frame": self._frame,
            "tensors": tensors,
            "outputs": (rgb, depth, alpha),
            "counter_event": counter_event,
            "chunks": chunks,
        }
        return rgb, depth, alpha

    def _reserve_host_counters(self, slots: int) -> None:
        """Pinned host rows for the deferred counter copies of one frame's
        camera chunks (sized before any copy of the frame is queued)."""
        if self._host_counters is None or self._host_counters.shape[0] < slots:
            self._host_counters = torch.zeros((max(slots, 8), 5), dtype=torch.int64, pin_memory=True)

    def _camera_chunks(self, b: int) -> list[tuple[int, int]]:
        """Camera ranges whose kept lists fit the memory budget (one range
        without a budget).  The per-camera size is learned from the counters
        of earlier renders; the first budgeted render uses one camera."""
        if self.list_budget_bytes is None:
            return [(0, b)]
        per = 1 if self._bytes_per_camera is None else max(
            1, min(b, int(self.list_budget_bytes // max(self._bytes_per_camera, 1.0))))
        return [(s, min(b, s + per)) for s in range(0, b, per)]

    def _render_range(self, tensors, outputs, s: int, e: int, *, allow_deferred: bool, cam_offset: int = 0,
                      slot: int = 0):
        """Training forward of cameras [cam_offset + s, cam_offset + e) into
        the outputs' rows [s, e) and the per-pixel state of those cameras'
        pixels; grows the capacity and re-renders on overflow (synchronously
        unless deferred checks apply)."""
        means, _, _, _, features, viewmats, intrinsics = tensors
        rgb, depth, alpha = (t[s:e] for t in outputs)
        c0, c1 = cam_offset + s, cam_offset + e
        device = means.device
        stream = torch.cuda.current_stream(device).cuda_stream
        for _attempt in range(8):
            scene, cams, outs, native_ws, options, state = self._structs(
                means, features, viewmats[c0:c1], intrinsics[c0:c1], rgb, depth, alpha, cam0=c0
            )
            selector = _native._c_i64(1)
            _native.check(
                self._lib.vgr_render_train(scene, cams, outs, native_ws, options, state, stream, selector),
                "render_train",
            )
            # Deferred only for camera ranges no larger than a checked one: a
            # wider range (a budget's chunk size learned from one camera)
            # is checked synchronously and grows the capacity first.
            if (allow_deferred and self.capacity_check == "deferred" and self._calibrated
                    and e - s <= self._calibrated_cameras):
                # Checked by the backward (or the next forward), which waits
                # only for this forward, not for the work queued after it.
                self._host_counters[slot].copy_(self._ws["counters"], non_blocking=True)
                counter_event = torch.cuda.Event()
                counter_event.record(torch.cuda.current_stream(device))
                return counter_event
            counters = self._ws["counters"].tolist()
            self.last_counters = {"visible_gaussians": counters[0], "tile_intersections": counters[1]}
            if counters[0] <= self._visible_capacity and counters[1] <= self._intersection_capacity:
                self._calibrated = True
                self._calibrated_cameras = max(self._calibrated_cameras, e - s)
                self._bytes_per_camera = (24.0 * counters[1] + 96.0 * counters[0]
                                          + 4.0 * means.shape[0] * (e - s)) / (e - s)
                return None
            self._visible_capacity = min(max(self._visible_capacity, int(counters[0] * self.headroom) + 1), _INT32_MAX)
            self._intersection_capacity = min(
                max(self._intersection_capacity, int(counters[1] * self.headroom) + 1), _INT32_MAX
            )
            if counters[1] > _INT32_MAX:
                raise RuntimeError("tile intersections exceed the int32 implementation limit")
            self._grow(device)
        raise RuntimeError("render_train: capacity did not converge")

    def check_capacity(self) -> None:
        """Deferred capacity check of the last forward: raises when it
        overflowed (its outputs and gradients are invalid), after growing the
        capacity so that rendering the frame again succeeds."""
        pending = self._pending
        event = pending.get("counter_event") if pending else None
        if event is None:
            return
        event.synchronize()
        pending["counter_event"] = None
        self._raise_on_overflow(len(pending.get("chunks", [(0, 0)])), f"frame {pending['frame']}")

    def _raise_on_overflow(self, slots: int, what: str) -> None:
        """Check the counters the deferred renders copied to the host (one
        row per camera chunk); grow and raise when any overflowed."""
        rows = self._host_counters[:slots].tolist()
        counters = [max(r[0] for r in rows), max(r[1] for r in rows)]
        last = rows[-1]
        self.last_counters = {"visible_gaussians": last[0], "tile_intersections": last[1]}
        if counters[0] <= self._visible_capacity and counters[1] <= self._intersection_capacity:
            return
        self._visible_capacity = min(max(self._visible_capacity, int(counters[0] * self.headroom) + 1), _INT32_MAX)
        self._intersection_capacity = min(
            max(self._intersection_capacity, int(counters[1] * self.headroom) + 1), _INT32_MAX
        )
        self._grow(self._pending["outputs"][0].device)
        self._calibrated = False
        raise RuntimeError(
            f"{what} overflowed the record or intersection capacity "
            f"({counters[0]} records, {counters[1]} intersections); its outputs are invalid. "
            "Capacity has been grown: render the frame again."
        )

    # -------------------------------------------------------------- backward
    def backward_native(self, frame: int, grad_rgb, grad_depth, grad_alpha):
        """Parameter gradients of the frame ``frame`` (the last forward)."""
        pending = self._pending
        if pending is None or pending["frame"] != frame:
            raise RuntimeError(
                "DifferentiableRenderer keeps one frame in flight: run the backward of a frame "
                "before rendering the next one"
            )
        self.check_capacity()
        means, log_scales, rotations, opacity_logits, features, viewmats, intrinsics = pending["tensors"]
        rgb, depth, alpha = pending["outputs"]
        device = means.device
        g = means.shape[0]
        if grad_rgb is None:
            grad_rgb = torch.zeros_like(rgb)
        grad_rgb = grad_rgb.contiguous()
        grad_depth = grad_depth.contiguous() if grad_depth is not None else None
        grad_alpha = grad_alpha.contiguous() if grad_alpha is not None else None
        chunks = pending.get("chunks", [(0, viewmats.shape[0])])
        params = _native.VgrTrainParams(
            log_scales=log_scales.data_ptr(), rotations=rotations.data_ptr(),
            opacity_logits=opacity_logits.data_ptr(),
        )
        stream = torch.cuda.current_stream(device).cuda_stream

        def backward_range(s: int, e: int, fwd):
            d = (torch.empty((g, 3), dtype=torch.float32, device=device),
                 torch.empty((g, 3), dtype=torch.float32, device=device),
                 torch.empty((g, 4), dtype=torch.float32, device=device),
                 torch.empty((g,), dtype=torch.float32, device=device),
                 torch.empty_like(features))
            scene, cams, outs, native_ws, options, state = self._structs(
                means, features, viewmats[s:e], intrinsics[s:e], *fwd, cam0=s
            )
            grads = _native.VgrOutputGrads(
                rgb=grad_rgb[s:e].data_ptr(),
                depth=grad_depth[s:e].data_ptr() if grad_depth is not None else None,
                alpha=grad_alpha[s:e].data_ptr() if grad_alpha is not None else None,
            )
            out = _native.VgrParamGrads(
                means=d[0].data_ptr(), log_scales=d[1].data_ptr(), rotations=d[2].data_ptr(),
                opacity_logits=d[3].data_ptr(), features=d[4].data_ptr(),
            )
            _native.check(
                self._lib.vgr_render_backward(scene, params, cams, outs, native_ws, options, state, grads, out,
                                              stream),
                "render_backward",
            )
            return d

        if len(chunks) == 1:
            s, e = chunks[0]
            return backward_range(s, e, (rgb[s:e], depth[s:e], alpha[s:e]))
        # Lists beyond the budget were not kept: recompute each chunk's lists
        # (its forward again, into scratch outputs: the same values bit for
        # bit, and the same per-pixel state) before its backward.
        totals = None
        tensors = pending["tensors"]
        per = max(e - s for s, e in chunks)
        scratch = (torch.empty((per,) + tuple(rgb.shape[1:]), dtype=rgb.dtype, device=device),
                   torch.empty((per,) + tuple(depth.shape[1:]), dtype=depth.dtype, device=device),
                   torch.empty((per,) + tuple(alpha.shape[1:]), dtype=alpha.dtype, device=device))
        self._reserve_host_counters(len(chunks))
        event = None
        for slot, (s, e) in enumerate(chunks):
            fwd = tuple(t[: e - s] for t in scratch)
            event = self._render_range(tensors, fwd, 0, e - s, allow_deferred=True, cam_offset=s,
                                       slot=slot) or event
            part = backward_range(s, e, fwd)
            totals = part if totals is None else tuple(t.add_(p) for t, p in zip(totals, part))
        if event is not None:
            event.synchronize()
            self._raise_on_overflow(len(chunks), f"the backward of frame {frame}")
        return totals

    @property
    def frame(self) -> int:
        return self._frame


class _RenderFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, renderer, means, log_scales, rotations, opacity_logits, features, viewmats, intrinsics):
        rgb, depth, alpha = renderer.forward_native(
            means.detach(), log_scales.detach(), rotations.detach(), opacity_logits.detach(),
            features.detach(), viewmats.detach(), intrinsics.detach(),
        )
        ctx.renderer = renderer
        ctx.frame = renderer.frame
        return rgb, depth, alpha

    @staticmethod
    def backward(ctx, grad_rgb, grad_depth, grad_alpha):
        grads = ctx.renderer.backward_native(ctx.frame, grad_rgb, grad_depth, grad_alpha)
        return (None, *grads, None, None)


class _PhotometricLoss(torch.autograd.Function):
    @staticmethod
    def forward(ctx, rgb, depth, target_rgb, target_depth, depth_weight):
        lib = _native.load_library()
        rgb_c, depth_c = rgb.contiguous(), depth.contiguous()
        t_rgb, t_depth = target_rgb.contiguous(), target_depth.contiguous()
        pixels = depth_c.numel()
        if rgb_c.numel() != 3 * pixels or t_rgb.shape != rgb_c.shape or t_depth.shape != depth_c.shape:
            raise ValueError("rgb [...,3], depth [...,1] and their targets must match")
        for t in (rgb_c, depth_c, t_rgb, t_depth):
            if t.dtype != torch.float32 or t.device.type != "cuda":
                raise ValueError("photometric_loss takes float32 CUDA tensors")
        loss = torch.empty((), dtype=torch.float32, device=rgb.device)
        grad_rgb = torch.empty_like(rgb_c)
        grad_depth = torch.empty_like(depth_c)
        stream = torch.cuda.current_stream(rgb.device).cuda_stream
        _native.check(
            lib.vgr_photometric_loss(rgb_c.data_ptr(), t_rgb.data_ptr(), depth_c.data_ptr(), t_depth.data_ptr(),
                                     pixels, float(depth_weight), loss.data_ptr(), grad_rgb.data_ptr(),
                                     grad_depth.data_ptr(), stream),
            "photometric_loss",
        )
        ctx.save_for_backward(grad_rgb, grad_depth)
        return loss

    @staticmethod
    def backward(ctx, grad_loss):
        grad_rgb, grad_depth = ctx.saved_tensors
        return grad_rgb * grad_loss, grad_depth * grad_loss, None, None, None


def photometric_loss(rgb: torch.Tensor, depth: torch.Tensor, target_rgb: torch.Tensor,
                     target_depth: torch.Tensor, depth_weight: float = 0.1) -> torch.Tensor:
    """``mean((rgb - target_rgb)^2) + depth_weight * mean(|depth - target_depth|)``
    (the depth term over pixels where both depths are finite, divided by the
    pixel count), forward and gradient in one CUDA pass."""
    return _PhotometricLoss.apply(rgb, depth, target_rgb, target_depth, depth_weight)
