"""GPU compositor of a Gaussian render layer and a dynamic mesh render layer.

Counterpart of src/isaacsim_gaussian_renderer/hybrid_compositor.py: same
function, arguments, validation and result type; the composite itself is one
CUDA kernel (``vgr_composite_gaussian_and_mesh``) that reads both layers once
and writes the four outputs, bit-identical to the reference's float32 tensor
expression.
"""

from __future__ import annotations

from dataclasses import dataclass

import torch

from . import _native


@dataclass(frozen=True)
class HybridComposite:
    """Straight-alpha RGB, alpha, depth, and front-layer selection tensors."""

    rgb: torch.Tensor
    alpha: torch.Tensor
    depth: torch.Tensor
    mesh_in_front: torch.Tensor


def _validate_layer(rgb: torch.Tensor, alpha: torch.Tensor, depth: torch.Tensor, name: str) -> None:
    if rgb.ndim != 4 or rgb.shape[-1] != 3 or not torch.is_floating_point(rgb):
        raise ValueError(f"{name}_rgb must be floating [B,H,W,3].")
    expected = (*rgb.shape[:3], 1)
    for tensor, suffix in ((alpha, "alpha"), (depth, "depth")):
        if tensor.shape != expected or not torch.is_floating_point(tensor):
            raise ValueError(f"{name}_{suffix} must be floating [B,H,W,1], got {tuple(tensor.shape)}.")
        if tensor.device != rgb.device:
            raise ValueError(f"{name}_{suffix} must share the RGB device.")


def composite_gaussian_and_mesh(
    gaussian_rgb: torch.Tensor,
    gaussian_alpha: torch.Tensor,
    gaussian_depth: torch.Tensor,
    mesh_rgb: torch.Tensor,
    mesh_alpha: torch.Tensor,
    mesh_depth: torch.Tensor,
    *,
    min_alpha: float = 1.0e-4,
    depth_epsilon: float = 1.0e-4,
) -> HybridComposite:
    """Depth-order and straight-alpha composite two GPU-resident render layers
    (RGB ``[B,H,W,3]``, alpha/depth ``[B,H,W,1]``; empty pixels are selected by
    alpha, not by a sentinel depth)."""
    _validate_layer(gaussian_rgb, gaussian_alpha, gaussian_depth, "gaussian")
    _validate_layer(mesh_rgb, mesh_alpha, mesh_depth, "mesh")
    if gaussian_rgb.shape != mesh_rgb.shape:
        raise ValueError("Gaussian and mesh RGB tensors must have equal shapes.")
    if gaussian_rgb.device != mesh_rgb.device:
        raise ValueError("Gaussian and mesh tensors must share one device.")
    if not 0.0 <= min_alpha <= 1.0:
        raise ValueError("min_alpha must be in [0, 1].")
    if depth_epsilon < 0.0:
        raise ValueError("depth_epsilon must be non-negative.")
    if gaussian_rgb.device.type != "cuda":
        raise ValueError("the hybrid compositor runs on CUDA tensors")
    layers = [t.to(torch.float32).contiguous() for t in
              (gaussian_rgb, gaussian_alpha, gaussian_depth, mesh_rgb, mesh_alpha, mesh_depth)]
    rgb = torch.empty_like(layers[0])
    alpha = torch.empty_like(layers[1])
    depth = torch.empty_like(layers[2])
    front = torch.empty(alpha.shape, dtype=torch.uint8, device=alpha.device)
    lib = _native.load_library()
    with torch.cuda.device(rgb.device):
        _native.check(
            lib.vgr_composite_gaussian_and_mesh(
                *(t.data_ptr() for t in layers), alpha.numel(), float(min_alpha), float(depth_epsilon),
                rgb.data_ptr(), alpha.data_ptr(), depth.data_ptr(), front.data_ptr(),
                torch.cuda.current_stream(rgb.device).cuda_stream,
            ),
            "composite_gaussian_and_mesh",
        )
    return HybridComposite(rgb=rgb, alpha=alpha, depth=depth, mesh_in_front=front.view(torch.bool))
