"""Shared helpers: render a scene with the CUDA backend and with the oracle."""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch

from oracle import camera as oracle_camera
from vgr_b200 import CustomCudaBackend, RendererService
from vgr_b200.workloads import CameraRig, SceneTensors


@dataclass
class GpuFrame:
    outputs: dict[str, torch.Tensor]
    counters: dict[str, int]
    backend: CustomCudaBackend
    service: RendererService


def render_gpu(
    scenes: list[tuple[int, SceneTensors]],
    rig: CameraRig,
    scene_ids: list[int],
    *,
    active_ids: list[int] | None = None,
    outputs: tuple[str, ...] = ("rgb", "depth", "alpha", "semantic_id"),
    **backend_kwargs,
) -> GpuFrame:
    device = torch.device("cuda")
    backend_kwargs.setdefault("output_srgb", False)
    backend = CustomCudaBackend(**backend_kwargs)
    service = RendererService(
        backend, height=rig.height, width=rig.width, outputs=outputs, max_views=rig.viewmats.shape[0]
    )
    service.initialize(stage=None, device=device)
    for sid, scene in scenes:
        service.load_scene(sid, **scene.to(device).as_kwargs())
    active = None if active_ids is None else torch.tensor(active_ids, dtype=torch.int64, device=device)
    out = service.render(
        rig.viewmats.to(device),
        rig.intrinsics.to(device),
        torch.tensor(scene_ids, dtype=torch.int64, device=device),
        active_camera_ids=active,
    )
    service.synchronize()
    counters = backend.read_counters()
    return GpuFrame({k: v.clone() for k, v in out.items()}, counters, backend, service)


def render_oracle(
    scenes: list[tuple[int, SceneTensors]],
    rig: CameraRig,
    scene_ids: list[int],
    *,
    active_ids: list[int] | None = None,
    with_tiles: bool = False,
    near_plane: float = 0.01,
    far_plane: float = 100.0,
    gaussian_support_sigma: float = 3.33,
    covariance_epsilon: float = 0.3,
    semantic_min_alpha: float = 0.01,
    rasterize_mode: str = "classic",
    tile_size: int = 16,
    output_srgb: bool = False,
    sh_degree: int | None = None,
    ray_gaussian_evaluation: bool = False,
    **_ignored,
):
    means = np.concatenate([s.means.numpy() for _, s in scenes])
    scales = np.concatenate([s.scales.numpy() for _, s in scenes])
    rotations = np.concatenate([s.rotations.numpy() for _, s in scenes])
    covariances = oracle_camera.precompute_covariances(scales, rotations)
    offsets = np.cumsum([0] + [s.means.shape[0] for _, s in scenes]).astype(np.int64)
    return oracle_camera.render(
        means=means,
        covariances=covariances,
        opacities=np.concatenate([s.opacities.numpy() for _, s in scenes]),
        features=np.concatenate([s.features.numpy() for _, s in scenes]),
        semantic_ids=np.concatenate([s.semantic_ids.numpy() for _, s in scenes]),
        registered_scene_ids=np.array([sid for sid, _ in scenes], dtype=np.int64),
        scene_offsets=offsets,
        viewmats=rig.viewmats.numpy(),
        intrinsics=rig.intrinsics.numpy(),
        camera_scene_ids=np.array(scene_ids, dtype=np.int64),
        height=rig.height,
        width=rig.width,
        active_ids=active_ids,
        near_plane=near_plane,
        far_plane=far_plane,
        support_sigma=gaussian_support_sigma,
        covariance_epsilon=covariance_epsilon,
        semantic_min_alpha=semantic_min_alpha,
        antialiased=rasterize_mode == "antialiased",
        tile_size=tile_size,
        output_srgb=output_srgb,
        sh_degree=-1 if sh_degree is None else sh_degree,
        with_tiles=with_tiles,
        ray_gaussian_evaluation=ray_gaussian_evaluation,
    )


def assert_bitwise_equal(gpu: np.ndarray, cpu: np.ndarray, name: str) -> None:
    gpu = np.asarray(gpu)
    cpu = np.asarray(cpu)
    assert gpu.shape == cpu.shape, (name, gpu.shape, cpu.shape)
    if gpu.dtype.kind == "f":
        same = (gpu.view(np.uint32) == cpu.view(np.uint32)) | (np.isnan(gpu) & np.isnan(cpu))
    else:
        same = gpu == cpu
    if not same.all():
        bad = np.argwhere(~same)
        first = tuple(bad[0])
        raise AssertionError(
            f"{name}: {bad.shape[0]} of {same.size} elements differ; first at {first}: "
            f"gpu={gpu[first]!r} cpu={cpu[first]!r}"
        )
