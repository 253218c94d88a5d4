"""Camera ingestion: USD camera world matrices -> OpenCV view matrices.

Counterpart of the Warp kernel ``fabric_world_to_opencv_viewmats``
(src/isaacsim_gaussian_renderer/fabric_camera_kernels.py:8-49) that the
reference's Isaac integration runs on zero-copy Fabric arrays: one CUDA
thread per camera (``vgr_world_to_opencv_viewmats``), writing row
``camera_indices[i]`` of the renderer's ``[B,4,4]`` view matrices.
"""

from __future__ import annotations

import torch

from . import _native


def world_to_opencv_viewmats(
    world_matrices: torch.Tensor,
    viewmats: torch.Tensor,
    camera_indices: torch.Tensor | None = None,
) -> int:
    """Convert USD row-vector world matrices ``[N,4,4]`` (float64) into
    OpenCV world->camera matrices, in place in ``viewmats [B,4,4]`` (float32).
    Returns the number of skipped out-of-range indices (synchronises)."""
    if world_matrices.dtype != torch.float64 or world_matrices.dim() != 3 or world_matrices.shape[1:] != (4, 4):
        raise ValueError("world_matrices must be float64 [N,4,4]")
    if viewmats.dtype != torch.float32 or viewmats.dim() != 3 or viewmats.shape[1:] != (4, 4):
        raise ValueError("viewmats must be float32 [B,4,4]")
    if not (world_matrices.is_cuda and viewmats.is_cuda and world_matrices.device == viewmats.device):
        raise ValueError("camera ingestion runs on one CUDA device")
    if not (world_matrices.is_contiguous() and viewmats.is_contiguous()):
        raise ValueError("world_matrices and viewmats must be contiguous")
    n = world_matrices.shape[0]
    if camera_indices is not None:
        if camera_indices.dtype != torch.int32 or camera_indices.shape != (n,) or camera_indices.device != viewmats.device:
            raise ValueError("camera_indices must be int32 [N] on the same device")
        camera_indices = camera_indices.contiguous()
    bad = torch.zeros((1,), dtype=torch.int32, device=viewmats.device)
    lib = _native.load_library()
    with torch.cuda.device(viewmats.device):
        _native.check(
            lib.vgr_world_to_opencv_viewmats(
                world_matrices.data_ptr(),
                None if camera_indices is None else camera_indices.data_ptr(),
                n, viewmats.data_ptr(), viewmats.shape[0], bad.data_ptr(),
                torch.cuda.current_stream(viewmats.device).cuda_stream,
            ),
            "world_to_opencv_viewmats",
        )
    return int(bad.item())
