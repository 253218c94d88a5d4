"""Dense mode (tile_size=1, the reference's per-pixel path) vs the CPU oracle.

Dense mode culls tile keys behind a per-tile optical-thickness depth cutoff
(every pixel of the tile has reached T <= 1e-4 before the first culled
record), so its images are the plain path's bit for bit; only the key count
drops.  Checked on a deep scene where most keys are culled, on a shallow one
where few are, through the backend (compact and non-compact) and through the
drop-in native module with the reference's per-pixel workspace.
"""

from __future__ import annotations

import math

import numpy as np
import pytest
import torch

from helpers import assert_bitwise_equal, render_gpu, render_oracle
from vgr_b200 import native_module
from vgr_b200.workloads import CameraRig, SceneTensors, orbit_cameras, pinhole, synthetic_scene

pytestmark = pytest.mark.gpu


def _deep_scene(count=40_000, seed=31) -> SceneTensors:
    # Stacked layers of large, fairly opaque Gaussians in front of the camera:
    # every pixel saturates within the first few layers.
    scene = synthetic_scene(count, seed=seed, mean_half_extent=1.0, log_scale_mean=-2.3, log_scale_std=0.2)
    gen = torch.Generator().manual_seed(seed)
    scene.means[:, 2] = torch.randint(0, 40, (count,), generator=gen).float() * 0.05
    scene.opacities.copy_(0.6 + 0.39 * torch.rand((count,), generator=gen))
    return scene


def _deep_rig(batch=2, width=96, height=80) -> CameraRig:
    view = torch.eye(4).repeat(batch, 1, 1)
    view[:, 2, 3] = 2.5
    if batch > 1:
        view[1, 0, 3] = 0.2
    return CameraRig(view.contiguous(), pinhole(batch, 70.0, 70.0, width / 2.0, height / 2.0), height, width)


def _compare_images(gpu, cpu):
    mapping = {"rgb": cpu.rgb, "depth": cpu.depth, "alpha": cpu.alpha, "semantic_id": cpu.semantic}
    for name, want in mapping.items():
        assert_bitwise_equal(gpu.outputs[name].cpu().numpy(), want, name)


@pytest.mark.parametrize("compact", [False, True])
def test_dense_mode_deep_scene_culls_and_matches_oracle(compact):
    scene, rig = _deep_scene(), _deep_rig()
    opts = {"tile_size": 1, "compact_projection_cache": compact, "deterministic": not compact}
    dense = render_gpu([(5, scene)], rig, [5, 5], **opts)
    plain = render_gpu([(5, scene)], rig, [5, 5], tile_size=16)
    cpu = render_oracle([(5, scene)], rig, [5, 5], tile_size=16)
    _compare_images(dense, cpu)
    _compare_images(plain, cpu)
    kept = dense.counters["tile_intersections"]
    full = plain.counters["tile_intersections"]
    assert full == cpu.intersections
    assert kept < 0.5 * full, (kept, full)  # the cutoff removes most keys here
    assert dense.counters["visible_gaussians"] <= plain.counters["visible_gaussians"]
    assert dense.counters["intersection_overflow"] == 0


def test_dense_mode_shallow_scene_matches_oracle():
    scene = synthetic_scene(20_000, seed=5, mean_half_extent=1.5, log_scale_mean=-3.5, sh_degree=2)
    rig = orbit_cameras(3, seed=3, radius=4.0, height_offset=0.8, width=100, height=72, focal=90.0)
    dense = render_gpu([(7, scene)], rig, [7] * 3, tile_size=1, sh_degree=2)
    cpu = render_oracle([(7, scene)], rig, [7] * 3, tile_size=16, sh_degree=2, with_tiles=True)
    _compare_images(dense, cpu)
    assert dense.counters["tile_intersections"] <= cpu.intersections


def test_dense_mode_repeat_and_antialiased():
    scene, rig = _deep_scene(20_000, seed=32), _deep_rig(batch=1, width=64, height=64)
    first = render_gpu([(5, scene)], rig, [5], tile_size=1, rasterize_mode="antialiased")
    second = render_gpu([(5, scene)], rig, [5], tile_size=1, rasterize_mode="antialiased")
    for name in first.outputs:
        assert torch.equal(first.outputs[name], second.outputs[name]), name
    cpu = render_oracle([(5, scene)], rig, [5], tile_size=16, rasterize_mode="antialiased")
    _compare_images(first, cpu)


def test_dense_mode_through_native_module():
    device = torch.device("cuda")
    mod = native_module.load_native_extension()
    scene, rig = _deep_scene(20_000, seed=33), _deep_rig()
    batch, height, width = 2, rig.height, rig.width
    s = scene.to(device)
    covariances = torch.empty((s.means.shape[0], 6), dtype=torch.float32, device=device)
    mod.precompute_covariances(s.scales, s.rotations, covariances)
    scene_tensors = [
        s.means, covariances, s.opacities, s.features, s.semantic_ids,
        torch.tensor([5], dtype=torch.int64, device=device),
        torch.tensor([0, s.means.shape[0]], dtype=torch.int64, device=device),
    ]
    cameras = [
        rig.viewmats.to(device).contiguous(),
        rig.intrinsics.to(device).contiguous(),
        torch.eye(4, device=device).repeat(batch, 1, 1).contiguous(),
        torch.full((batch,), 5, dtype=torch.int64, device=device),
        torch.empty((0,), dtype=torch.int64, device=device),
    ]
    outputs = [
        torch.empty((batch, height, width, 3), dtype=torch.float32, device=device),
        torch.empty((batch, height, width, 1), dtype=torch.float32, device=device),
        torch.empty((batch, height, width, 1), dtype=torch.float32, device=device),
        torch.empty((batch, height, width, 1), dtype=torch.int64, device=device),
    ]
    pixels = batch * height * width  # the reference sizes tile ranges per pixel at tile_size 1
    visible, isect = batch * s.means.shape[0], 2_000_000
    f32, i32 = torch.float32, torch.int32
    ws = [
        torch.empty((visible, 2), dtype=f32, device=device),
        torch.empty((visible, 3), dtype=f32, device=device),
        torch.empty((visible,), dtype=f32, device=device),
        torch.empty((visible,), dtype=f32, device=device),
        torch.empty((visible,), dtype=i32, device=device),
        torch.empty((visible,), dtype=i32, device=device),
        torch.empty((visible, 2), dtype=i32, device=device),
        torch.empty((isect,), dtype=torch.uint64, device=device),
        torch.empty((isect,), dtype=torch.uint64, device=device),
        torch.empty((isect,), dtype=i32, device=device),
        torch.empty((isect,), dtype=i32, device=device),
        torch.empty((pixels,), dtype=i32, device=device),
        torch.empty((pixels,), dtype=i32, device=device),
        torch.zeros((5,), dtype=torch.int64, device=device),
        torch.empty((mod.radix_sort_double_buffer_temp_bytes(isect, pixels),), dtype=torch.uint8, device=device),
    ]
    ws += [torch.empty((1,), dtype=f32, device=device) for _ in range(24 - len(ws))]
    mod.render(scene_tensors, cameras, outputs, ws, height, width, s.means.shape[0], 0.01, 100.0, 3.33, 0.3,
               False, 0.01, False, 1, 4096, 64, True, False, False, False, False, True, False)
    torch.cuda.synchronize()
    cpu = render_oracle([(5, scene)], rig, [5, 5], tile_size=16)
    for got, want, name in zip(outputs, (cpu.rgb, cpu.depth, cpu.alpha, cpu.semantic),
                               ("rgb", "depth", "alpha", "semantic")):
        assert_bitwise_equal(got.cpu().numpy(), want, name)
    counters = ws[13].cpu().tolist()
    assert 0 < counters[1] < cpu.intersections
    assert math.isfinite(float(outputs[0].sum()))
