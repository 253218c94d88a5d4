"""Exact-ray evaluation mode (ray_gaussian_evaluation=True) vs the CPU oracle.

The projection computes the camera-space precision and the ray-ellipse cull
in double with explicit round-to-nearest operations, and the compositor
evaluates each pixel ray's Mahalanobis distance in float in the oracle's
operation order, so the comparison is bit-exact: outputs, counters, per-tile
counts and sorted Gaussian lists (renderer_cuda.cu:795-948,2190-2270 is the
reference equation; the 16-pixel tile bins as 32 pixels, 2670-2676).
"""

from __future__ import annotations

import math

import numpy as np
import pytest
import torch

from helpers import assert_bitwise_equal, render_gpu, render_oracle
from vgr_b200 import CustomCudaBackend, RendererService, native_module
from vgr_b200.ragged import RaggedBatch
from vgr_b200.workloads import CameraRig, look_at_viewmats, orbit_cameras, pinhole, synthetic_scene

pytestmark = pytest.mark.gpu


def _compare(gpu, cpu, outputs=("rgb", "depth", "alpha", "semantic_id")):
    mapping = {"rgb": cpu.rgb, "depth": cpu.depth, "alpha": cpu.alpha, "semantic_id": cpu.semantic}
    for name in outputs:
        assert_bitwise_equal(gpu.outputs[name].cpu().numpy(), mapping[name], name)
    assert gpu.counters["visible_gaussians"] == cpu.visible
    assert gpu.counters["tile_intersections"] == cpu.intersections
    assert gpu.counters["active_tiles"] == cpu.active_tiles
    assert gpu.counters["visible_overflow"] == 0
    assert gpu.counters["intersection_overflow"] == 0


def _sorted_gids(frame) -> np.ndarray:
    ws = frame.backend.workspace
    n = frame.counters["tile_intersections"]
    values = ws["values_out"][:n].long()
    gids = ws["records"].view(torch.int32)[:, 7]
    return gids[values].cpu().numpy()


def _batch4():
    scene = synthetic_scene(20_000, seed=5, mean_half_extent=1.5, log_scale_mean=-3.5)
    rig = orbit_cameras(4, seed=3, radius=4.0, height_offset=0.8, width=96, height=80, focal=90.0)
    return scene, rig


@pytest.mark.parametrize("tile_size", [4, 8, 16])
def test_exact_ray_bitwise(tile_size):
    scene, rig = _batch4()
    gpu = render_gpu([(7, scene)], rig, [7] * 4, tile_size=tile_size, ray_gaussian_evaluation=True)
    cpu = render_oracle([(7, scene)], rig, [7] * 4, tile_size=tile_size, with_tiles=True,
                        ray_gaussian_evaluation=True)
    _compare(gpu, cpu)
    assert_bitwise_equal(_sorted_gids(gpu), cpu.sorted_gaussian_ids, "sorted gaussian ids")
    starts = gpu.backend.workspace["tile_starts"].cpu().numpy()
    ends = gpu.backend.workspace["tile_ends"].cpu().numpy()
    bins = cpu.tile_counts.shape[0]
    assert_bitwise_equal((ends[:bins] - starts[:bins]).astype(np.int32), cpu.tile_counts, "per-tile counts")
    # Exact-ray and screen-space images differ (the modes are not aliases).
    screen = render_oracle([(7, scene)], rig, [7] * 4, tile_size=tile_size)
    assert np.abs(screen.rgb - cpu.rgb).max() > 1e-3


def test_exact_ray_sh3_spatial_layout_rgb_only():
    # Spatial layout's chunk frustum test is derived from the screen-space
    # cull; in exact-ray mode no chunk is skipped and ids follow the remap.
    scenes = [(4, synthetic_scene(30_000, seed=93, mean_half_extent=5.0, log_scale_mean=-3.0, sh_degree=3))]
    eyes = torch.tensor([[0.0, 0.5, 0.0], [3.0, 0.0, -2.0], [0.5, 1.0, 0.5]])
    targets = torch.tensor([[5.0, 0.0, 0.0], [3.0, 0.0, 5.0], [-4.0, 0.0, 0.0]])
    rig = CameraRig(look_at_viewmats(eyes, targets), pinhole(3, 70.0, 70.0, 48.0, 32.0), 64, 96)
    ids = [4, 4, 4]
    for outputs in (("rgb",), ("rgb", "depth", "alpha", "semantic_id")):
        gpu = render_gpu(scenes, rig, ids, sh_degree=3, spatial_layout=True, ray_gaussian_evaluation=True,
                         outputs=outputs)
        cpu = render_oracle(scenes, rig, ids, sh_degree=3, ray_gaussian_evaluation=True)
        _compare(gpu, cpu, outputs)


def test_exact_ray_near_camera_and_degenerate_ellipses():
    # Gaussians straddling the image edges and close to the near plane give
    # unbounded or very large ray ellipses (whole-image fallback), plus
    # needle-thin Gaussians: every branch of the ellipse cull.
    gen = torch.Generator().manual_seed(17)
    scene = synthetic_scene(4_000, seed=17, mean_half_extent=1.0, log_scale_mean=-2.5)
    scene.means[:400, 2] = torch.rand((400,), generator=gen) * 0.3 - 3.6  # just past the near plane
    scene.scales[400:600, 0] = 1e-4
    scene.scales[400:600, 1] = 0.5
    scene.opacities[600:700] = 1.0
    view = torch.eye(4).repeat(2, 1, 1)
    view[:, 2, 3] = 3.7
    view[1, 0, 3] = 0.4
    rig = CameraRig(view.contiguous(), pinhole(2, 60.0, 60.0, 40.0, 30.0), 60, 80)
    gpu = render_gpu([(2, scene)], rig, [2, 2], tile_size=8, ray_gaussian_evaluation=True, near_plane=0.05)
    cpu = render_oracle([(2, scene)], rig, [2, 2], tile_size=8, with_tiles=True, ray_gaussian_evaluation=True,
                        near_plane=0.05)
    _compare(gpu, cpu)
    assert_bitwise_equal(_sorted_gids(gpu), cpu.sorted_gaussian_ids, "sorted gaussian ids")


def test_exact_ray_mode_switch_after_allocation():
    # Turning exact-ray mode on after a screen-space frame grows the record
    # storage for the extension records; turning it off again renders the
    # screen-space frame unchanged.
    scene, rig = _batch4()
    device = torch.device("cuda")
    backend = CustomCudaBackend(output_srgb=False, tile_size=8)
    service = RendererService(backend, height=rig.height, width=rig.width, max_views=4)
    service.initialize(stage=None, device=device)
    service.load_scene(7, **scene.to(device).as_kwargs())
    args = (rig.viewmats.to(device), rig.intrinsics.to(device), torch.full((4,), 7, dtype=torch.int64, device=device))
    screen = {k: v.clone() for k, v in service.render(*args).items()}
    backend.ray_gaussian_evaluation = True
    ray = {k: v.clone() for k, v in service.render(*args).items()}
    backend.ray_gaussian_evaluation = False
    again = service.render(*args)
    cpu = render_oracle([(7, scene)], rig, [7] * 4, tile_size=8, ray_gaussian_evaluation=True)
    assert_bitwise_equal(ray["rgb"].cpu().numpy(), cpu.rgb, "rgb")
    for name in screen:
        assert torch.equal(screen[name], again[name]), name
    with pytest.raises(ValueError, match="incompatible"):
        backend.rasterize_mode = "antialiased"
        backend.ray_gaussian_evaluation = True


def test_exact_ray_ragged_batch_matches_oracle_per_camera():
    resolutions = [(64, 48), (40, 56), (33, 17), (72, 96)]
    scenes = [(3, synthetic_scene(6_000, seed=81, mean_half_extent=1.2, log_scale_mean=-3.4))]
    device = torch.device("cuda")
    backend = CustomCudaBackend(output_srgb=False, tile_size=16, ray_gaussian_evaluation=True)
    service = RendererService(backend, height=64, width=64, max_views=1)
    service.initialize(stage=None, device=device)
    service.load_scene(3, **scenes[0][1].to(device).as_kwargs())
    ragged = RaggedBatch(backend, [h for h, _ in resolutions], [w for _, w in resolutions], tile_size=16)
    angle = torch.linspace(0.0, 5.0, len(resolutions), dtype=torch.float64)
    eyes = torch.stack((3.5 * torch.cos(angle), torch.full_like(angle, 0.7), 3.5 * torch.sin(angle)), dim=1)
    view = look_at_viewmats(eyes, torch.zeros((len(resolutions), 3), dtype=torch.float64))
    intr = torch.cat([pinhole(1, 0.9 * w, 0.9 * w, w / 2.0, h / 2.0) for h, w in resolutions])
    ids = torch.full((len(resolutions),), 3, dtype=torch.int64, device=device)
    outputs = ragged.outputs()
    ragged.calibrate(view.to(device), intr.to(device), ids, outputs)
    torch.cuda.synchronize()
    for c, (h, w) in enumerate(resolutions):
        rig = CameraRig(view[c:c + 1].contiguous(), intr[c:c + 1].contiguous(), h, w)
        # The ragged form bins in its own 16-pixel tiles; the images do not
        # depend on the bin size.
        cpu = render_oracle(scenes, rig, [3], tile_size=8, ray_gaussian_evaluation=True)
        for name, want in (("rgb", cpu.rgb), ("depth", cpu.depth), ("alpha", cpu.alpha), ("semantic_id", cpu.semantic)):
            assert_bitwise_equal(ragged.view(outputs, name, c).cpu().numpy(), want[0], f"camera {c} {name}")


def _reference_workspace(visible: int, intersections: int, tiles: int, device, ray_rows: int):
    mod = native_module.load_native_extension()
    sort_bytes = mod.sort_temp_bytes(intersections, tiles)
    f32, i32 = torch.float32, torch.int32
    ws = [
        torch.empty((visible, 2), dtype=f32, device=device),
        torch.empty((visible, 3), dtype=f32, device=device),
        torch.empty((visible,), dtype=f32, device=device),
        torch.empty((visible,), dtype=f32, device=device),
        torch.empty((visible,), dtype=i32, device=device),
        torch.empty((visible,), dtype=i32, device=device),
        torch.empty((visible, 2), dtype=i32, device=device),
        torch.empty((intersections,), dtype=torch.uint64, device=device),
        torch.empty((intersections,), dtype=torch.uint64, device=device),
        torch.empty((intersections,), dtype=i32, device=device),
        torch.empty((intersections,), dtype=i32, device=device),
        torch.empty((tiles,), dtype=i32, device=device),
        torch.empty((tiles,), dtype=i32, device=device),
        torch.zeros((5,), dtype=torch.int64, device=device),
        torch.empty((sort_bytes,), dtype=torch.uint8, device=device),
    ]
    ws += [torch.empty((0,), dtype=i32, device=device) for _ in range(22 - len(ws))]
    ws += [torch.empty((ray_rows, 6), dtype=f32, device=device), torch.empty((ray_rows, 4), dtype=f32, device=device)]
    return ws


def test_exact_ray_through_native_module():
    device = torch.device("cuda")
    mod = native_module.load_native_extension()
    scene = synthetic_scene(8_000, seed=101, mean_half_extent=1.5, log_scale_mean=-3.5)
    rig = orbit_cameras(3, seed=5, radius=4.0, height_offset=0.5, width=96, height=64, focal=80.0)
    batch, height, width, tile = 3, rig.height, rig.width, 16
    s = scene.to(device)
    covariances = torch.empty((s.means.shape[0], 6), dtype=torch.float32, device=device)
    mod.precompute_covariances(s.scales, s.rotations, covariances)
    scene_tensors = [
        s.means, covariances, s.opacities, s.features, s.semantic_ids,
        torch.tensor([7], dtype=torch.int64, device=device),
        torch.tensor([0, s.means.shape[0]], dtype=torch.int64, device=device),
    ]
    cameras = [
        rig.viewmats.to(device).contiguous(),
        rig.intrinsics.to(device).contiguous(),
        torch.eye(4, device=device).repeat(batch, 1, 1).contiguous(),
        torch.full((batch,), 7, dtype=torch.int64, device=device),
        torch.empty((0,), dtype=torch.int64, device=device),
    ]
    outputs = [
        torch.empty((batch, height, width, 3), dtype=torch.float32, device=device),
        torch.empty((batch, height, width, 1), dtype=torch.float32, device=device),
        torch.empty((batch, height, width, 1), dtype=torch.float32, device=device),
        torch.empty((batch, height, width, 1), dtype=torch.int64, device=device),
    ]
    tiles = batch * math.ceil(height / 32) * math.ceil(width / 32)  # 16-pixel tiles bin as 32
    visible = batch * s.means.shape[0]
    args = (height, width, s.means.shape[0], 0.01, 100.0, 3.33, 0.3, False, 0.01, True, tile, 4096, 64,
            False, False, False, False, True, True, False)
    small = _reference_workspace(visible, 400_000, tiles, device, ray_rows=1)
    with pytest.raises(RuntimeError, match="ray-precision workspace is too small"):
        mod.render(scene_tensors, cameras, outputs, small, *args)
    ws = _reference_workspace(visible, 400_000, tiles, device, ray_rows=visible)
    mod.render(scene_tensors, cameras, outputs, ws, *args)
    torch.cuda.synchronize()
    cpu = render_oracle([(7, scene)], CameraRig(rig.viewmats, rig.intrinsics, height, width), [7] * batch,
                        ray_gaussian_evaluation=True, with_tiles=True)
    for got, want, name in zip(outputs, (cpu.rgb, cpu.depth, cpu.alpha, cpu.semantic),
                               ("rgb", "depth", "alpha", "semantic")):
        assert_bitwise_equal(got.cpu().numpy(), want, name)
    counters = ws[13].cpu().tolist()
    assert counters[0] == cpu.visible and counters[1] == cpu.intersections
    assert_bitwise_equal((ws[12] - ws[11]).cpu().numpy().astype(np.int32), cpu.tile_counts, "tile counts")
    # The precision terms are mirrored into the reference's workspace slots
    # 22/23 (record order), equal to the extension records.
    prec = ws[22][: counters[0]].cpu()
    pm = ws[23][: counters[0]].cpu()
    assert torch.isfinite(prec).all() and torch.isfinite(pm).all()
    assert (prec[:, 0] > 0).all() and (prec[:, 3] > 0).all() and (prec[:, 5] > 0).all()  # P is positive definite

