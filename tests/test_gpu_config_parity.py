"""Parity at the full shapes of the configured workloads.

Every check renders the workload's own scene at its own resolution (the
seeded synthetic stand-ins of the five configurations) and compares a
bounded sample of its cameras or rays with the oracle, so the CPU side
finishes in seconds:

* batched: the 1M-Gaussian SH3 scene, four of the 64 orbit cameras at
  640x480 rendered as the active subset of the full 64-camera batch, in both
  ordering modes; bit for bit (RGB, depth, alpha, semantic, counters);
* ragged: all eight scenes (9.1M Gaussians) registered, one camera of each
  resolution (128x128, 160x120, 320x240) over the 100k, 1M and 3M scenes
  as one ragged submission; bit for bit per camera;
* differentiable: the 500k-Gaussian SH3 training scene, two of the sixteen
  512x512 cameras, through the training forward; bit for bit against the
  oracle given the forward's own activated covariances and opacities (the
  activations themselves are checked against float64 in
  test_differentiable.py);
* LiDAR: the 2M-Gaussian scene, sensor 0, every 256th ray of its 262,144,
  against the float64 LiDAR oracle: hit/miss agreement >= 99.8 % and range
  within 1e-4 m where both hit.
"""

from __future__ import annotations

import os

import numpy as np
import pytest
import torch

from helpers import assert_bitwise_equal, render_gpu, render_oracle
from oracle import camera as oc
from oracle import lidar as ol
from vgr_b200.workloads import CameraRig, batched_workload, lidar_workload, ragged_workload, training_workload

pytestmark = pytest.mark.gpu


def _compare_cameras(gpu: dict, cpu, cameras: list[int]) -> None:
    pairs = (("rgb", cpu.rgb), ("depth", cpu.depth), ("alpha", cpu.alpha), ("semantic_id", cpu.semantic))
    for name, want in pairs:
        got = gpu[name].cpu().numpy()
        assert_bitwise_equal(got[cameras], np.asarray(want)[cameras], name)


@pytest.mark.parametrize("deterministic", [True, False])
def test_batched_1m_sh3_four_of_64_cameras(deterministic):
    scene, rig = batched_workload()
    active = [0, 21, 42, 63]
    ids = [0] * rig.viewmats.shape[0]
    frame = render_gpu([(0, scene)], rig, ids, active_ids=active, sh_degree=3, deterministic=deterministic)
    cpu = render_oracle([(0, scene)], rig, ids, active_ids=active, sh_degree=3)
    _compare_cameras(frame.outputs, cpu, active)
    assert frame.counters["visible_gaussians"] == cpu.visible
    assert frame.counters["tile_intersections"] == cpu.intersections
    assert frame.counters["visible_overflow"] == frame.counters["intersection_overflow"] == 0


def test_ragged_nine_cameras_over_the_100k_1m_3m_scenes():
    from vgr_b200 import CustomCudaBackend, RendererService
    from vgr_b200.ragged import RaggedBatch

    work = ragged_workload(frames=1)
    cams = []
    for scene_id in (0, 4, 7):  # 100k, 1M and 3M Gaussians
        for res in ((128, 128), (120, 160), (240, 320)):
            cams.append(next(c for c in range(len(work.heights))
                             if int(work.scene_ids[c]) == scene_id and (work.heights[c], work.widths[c]) == res))
    device = torch.device("cuda")
    backend = CustomCudaBackend(sh_degree=3, output_srgb=False)
    holder = RendererService(backend, height=16, width=16, max_views=1)
    holder.initialize(stage=None, device=device)
    for sid, scene in work.scenes:
        holder.load_scene(sid, **scene.to(device).as_kwargs())
    heights = [work.heights[c] for c in cams]
    widths = [work.widths[c] for c in cams]
    ragged = RaggedBatch(backend, heights, widths)
    outputs = ragged.outputs()
    view = work.viewmats[0][cams].contiguous().to(device)
    intr = work.intrinsics[cams].contiguous().to(device)
    ids = work.scene_ids[cams].contiguous().to(device)
    counters = ragged.calibrate(view, intr, ids, outputs)
    ragged.render(view, intr, ids, outputs)
    torch.cuda.synchronize()
    scenes = [s for _, s in work.scenes]
    cpu = oc.render(
        means=np.concatenate([s.means.numpy() for s in scenes]),
        covariances=oc.precompute_covariances(np.concatenate([s.scales.numpy() for s in scenes]),
                                              np.concatenate([s.rotations.numpy() for s in scenes])),
        opacities=np.concatenate([s.opacities.numpy() for s in scenes]),
        features=np.concatenate([s.features.numpy() for s in scenes]),
        semantic_ids=np.concatenate([s.semantic_ids.numpy() for s in scenes]),
        registered_scene_ids=np.array([sid for sid, _ in work.scenes]),
        scene_offsets=np.cumsum([0] + [s.means.shape[0] for s in scenes]),
        viewmats=view.cpu().numpy(), intrinsics=intr.cpu().numpy(), camera_scene_ids=ids.cpu().numpy(),
        height=max(heights), width=max(widths), sh_degree=3, threads=os.cpu_count() or 1,
        ragged=dict(widths=widths, heights=heights,
                    tile_offsets=np.cumsum([0] + [-(-h // 16) * -(-w // 16) for h, w in zip(heights, widths)]),
                    pixel_offsets=np.cumsum([0] + [h * w for h, w in zip(heights, widths)])),
    )
    assert ragged.tile_size == 16
    for name, want in (("rgb", cpu.rgb), ("depth", cpu.depth[:, None]), ("alpha", cpu.alpha[:, None]),
                       ("semantic_id", cpu.semantic[:, None])):
        assert_bitwise_equal(outputs[name].cpu().numpy(), want, name)
    assert counters["visible_gaussians"] == cpu.visible
    assert counters["tile_intersections"] == cpu.intersections
    holder.shutdown()


def test_training_forward_500k_sh3_two_of_16_cameras():
    from vgr_b200.differentiable import DifferentiableRenderer

    work = training_workload()
    rig = work.rig
    pick = [0, 9]
    names = ("means", "log_scales", "rotations", "opacity_logits", "features")
    device = torch.device("cuda")
    params = [work.params[k].to(device) for k in names]
    view = rig.viewmats[pick].contiguous().to(device)
    intr = rig.intrinsics[pick].contiguous().to(device)
    renderer = DifferentiableRenderer(height=rig.height, width=rig.width, sh_degree=3, device=device)
    rgb, depth, alpha = renderer.forward_native(*params, view, intr)
    torch.cuda.synchronize()
    covariances = renderer._ws["covariances"].cpu().numpy()
    opacities = renderer._ws["opacities"].cpu().numpy()
    sub = CameraRig(rig.viewmats[pick].contiguous(), rig.intrinsics[pick].contiguous(), rig.height, rig.width)
    cpu = oc.render(
        means=work.params["means"].numpy(), covariances=covariances, opacities=opacities,
        features=work.params["features"].numpy(),
        semantic_ids=np.zeros(work.params["means"].shape[0], dtype=np.int64),
        registered_scene_ids=[0], scene_offsets=[0, work.params["means"].shape[0]],
        viewmats=sub.viewmats.numpy(), intrinsics=sub.intrinsics.numpy(), camera_scene_ids=[0, 0],
        height=sub.height, width=sub.width, sh_degree=3, threads=os.cpu_count() or 1,
    )
    assert_bitwise_equal(rgb.cpu().numpy(), cpu.rgb, "rgb")
    assert_bitwise_equal(depth.cpu().numpy(), cpu.depth, "depth")
    assert_bitwise_equal(alpha.cpu().numpy(), cpu.alpha, "alpha")


def test_lidar_2m_scene_sensor0_ray_subset():
    from test_gpu_lidar_parity import _gpu_render

    work = lidar_workload()  # 2M Gaussians, 64 sensors x 128 x 2048 rays
    stride = 256
    scene = {
        "means": work.means.double().numpy(), "scales": work.scales.double().numpy(),
        "rotations": work.rotations.double().numpy(), "opacities": work.opacities.double().numpy(),
        "semantic_ids": work.semantic_ids.numpy(), "reflectivity": work.reflectivity.double().numpy(),
        "surface_confidence": None,
    }
    case = {
        "scenes": {0: scene},
        "rays": work.ray_directions.double().numpy()[::stride].copy(),
        "times": work.time_offsets_ns.numpy()[::stride].copy(),
        "sensors": work.sensor_to_world.double().numpy()[:1].copy(),
        "scene_ids": np.array([0]),
        "kwargs": {"returns": 1},
    }
    config = ol.LidarConfig(far_plane_m=80.0)
    want = ol.render(case["scenes"], case["rays"], case["times"], case["sensors"], case["scene_ids"], returns=1,
                     config=config, threads=os.cpu_count() or 1)
    got, counters = _gpu_render(case, far_plane_m=80.0)
    assert counters["returns"] > 100
    agree = (got["valid"] == want["valid"]).mean()
    assert agree >= 0.998, agree
    both = got["valid"] & want["valid"]
    np.testing.assert_allclose(got["range_m"][both], want["range_m"][both], rtol=0, atol=1e-4)
    assert (got["semantic_id"][both] == want["semantic_id"][both]).mean() >= 0.998
