"""The drop-in native modules, called the way the reference's backends call
the reference extensions (cuda_backend.py, cuda_lidar_backend.py:302-366 and
:181-233): reference-shaped tensor lists in, reference-shaped results out.

Camera: ``native_module.render`` with the 7 scene / 5 camera / 4 output /
24 workspace tensors, against the bit-exact CPU oracle.  LiDAR:
``lidar_native_module`` build -> pack -> render on the reference's golden
cases, against the golden outputs.
"""

from __future__ import annotations

import math

import numpy as np
import pytest
import torch

from golden import lidar_cases
from helpers import assert_bitwise_equal, render_oracle
from vgr_b200 import native_module
from vgr_b200.cuda_lidar_backend import CudaLidarBackend
from vgr_b200.lidar_native_module import load_lidar_extension
from vgr_b200.workloads import CameraRig, orbit_cameras, synthetic_scene

pytestmark = pytest.mark.gpu


def _reference_workspace(visible: int, intersections: int, tiles: int, device) -> list[torch.Tensor]:
    mod = native_module.load_native_extension()
    sort_bytes = mod.radix_sort_double_buffer_temp_bytes(intersections, tiles)
    ws = [
        torch.empty((visible, 2), dtype=torch.float32, device=device),
        torch.empty((visible, 3), dtype=torch.float32, device=device),
        torch.empty((visible,), dtype=torch.float32, device=device),
        torch.empty((visible,), dtype=torch.float32, device=device),
        torch.empty((visible,), dtype=torch.int32, device=device),
        torch.empty((visible,), dtype=torch.int32, device=device),
        torch.empty((visible, 2), dtype=torch.int32, device=device),
        torch.empty((intersections,), dtype=torch.uint64, device=device),
        torch.empty((intersections,), dtype=torch.uint64, device=device),
        torch.empty((intersections,), dtype=torch.int32, device=device),
        torch.empty((intersections,), dtype=torch.int32, device=device),
        torch.empty((tiles,), dtype=torch.int32, device=device),
        torch.empty((tiles,), dtype=torch.int32, device=device),
        torch.zeros((5,), dtype=torch.int64, device=device),
        torch.empty((sort_bytes,), dtype=torch.uint8, device=device),
    ]
    ws += [torch.empty((0,), dtype=torch.int32, device=device) for _ in range(24 - len(ws))]
    return ws


def test_camera_native_module_render_matches_oracle():
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
    tiles = batch * math.ceil(height / tile) * math.ceil(width / tile)
    ws = _reference_workspace(batch * s.means.shape[0], 400_000, tiles, device)
    selector = mod.render(
        scene_tensors, cameras, outputs, ws, height, width, s.means.shape[0], 0.01, 100.0, 3.33, 0.3,
        False, 0.01, False, tile, 4096, 64, False, False, False, False, True, True, False,
    )
    torch.cuda.synchronize()
    assert selector in (0, 1)
    cpu = render_oracle([(7, scene)], CameraRig(rig.viewmats, rig.intrinsics, height, width), [7] * batch)
    for got, want, name in zip(outputs, (cpu.rgb, cpu.depth, cpu.alpha, cpu.semantic), ("rgb", "depth", "alpha", "semantic")):
        assert_bitwise_equal(got.cpu().numpy(), want, name)
    counters = ws[13].cpu().tolist()
    assert counters[0] == cpu.visible and counters[1] == cpu.intersections
    # Reference workspace mirrors of the visible records.
    ids = ws[5][: counters[0]].cpu()
    assert ids.min() >= 0 and ids.max() < s.means.shape[0]
    assert torch.unique(ws[4][: counters[0]].cpu()).tolist() == [0, 1, 2]


def _f32(a, device):
    return torch.as_tensor(np.asarray(a), dtype=torch.float32).contiguous().to(device)


def _render_through_module(case, packet):
    """The reference CudaLidarBackend's build/pack/render sequence."""
    device = torch.device("cuda")
    mod = load_lidar_extension()
    defaults = CudaLidarBackend()
    descriptors = torch.zeros((8, 14), dtype=torch.int64, device=device)
    counters = torch.zeros((12,), dtype=torch.int64, device=device)
    empty = torch.empty((0,), dtype=torch.float32, device=device)
    keep = []
    slots = {}
    for slot, (sid, sc) in enumerate(case["scenes"].items()):
        means = _f32(sc["means"], device)
        scales = _f32(sc["scales"], device)
        rotations = _f32(sc["rotations"], device)
        opacities = _f32(sc["opacities"], device)
        semantic = torch.as_tensor(sc["semantic_ids"], dtype=torch.int64).to(device)
        refl = empty if sc["reflectivity"] is None else _f32(sc["reflectivity"], device)
        conf = empty if sc["surface_confidence"] is None else _f32(sc["surface_confidence"], device)
        count = means.shape[0]
        leaf_count = math.ceil(count / packet)
        leaf_capacity = 1 << (leaf_count - 1).bit_length()
        sorted_indices = torch.empty((count,), dtype=torch.int32, device=device)
        node_bounds = torch.empty((2 * leaf_capacity - 1, 6), dtype=torch.float32, device=device)
        build = [
            torch.empty((count,), dtype=torch.uint64, device=device),
            torch.empty((count,), dtype=torch.uint64, device=device),
            torch.arange(count, dtype=torch.int32, device=device),
            sorted_indices,
            torch.empty((mod.sort_temp_bytes(count),), dtype=torch.uint8, device=device),
            torch.stack((means.amin(dim=0), means.amax(dim=0))).contiguous(),
            node_bounds,
        ]
        mod.build_scene_lbvh([means, scales, rotations], build, packet, leaf_count, leaf_capacity,
                             defaults.support_sigma, defaults.planarity_ratio_max)
        mod.pack_scene_descriptor(descriptors, slot, sid,
                                  [means, scales, rotations, opacities, semantic, refl, conf, sorted_indices,
                                   node_bounds], leaf_count, leaf_capacity)
        keep.append((means, scales, rotations, opacities, semantic, refl, conf, sorted_indices, node_bounds))
        slots[sid] = slot
    sensors = _f32(case["sensors"], device)
    batch = sensors.shape[0]
    rays = _f32(case["rays"], device)
    returns = case["kwargs"]["returns"]
    scene_to_world = (
        _f32(case["kwargs"]["scene_to_world"], device)
        if "scene_to_world" in case["kwargs"]
        else torch.eye(4, device=device).repeat(batch, 1, 1).contiguous()
    )
    active = (
        torch.as_tensor(case["kwargs"]["active_sensor_ids"], dtype=torch.int64).to(device)
        if "active_sensor_ids" in case["kwargs"]
        else torch.arange(batch, dtype=torch.int64, device=device)
    )
    inputs = [rays, torch.as_tensor(case["times"], dtype=torch.int64).to(device), sensors, scene_to_world,
              torch.as_tensor(case["scene_ids"], dtype=torch.int64).to(device), active]
    r = rays.shape[0]
    outputs = [
        torch.empty((batch, r, returns), dtype=torch.float32, device=device),
        torch.empty((batch, r, returns, 3), dtype=torch.float32, device=device),
        torch.empty((batch, r, returns), dtype=torch.float32, device=device),
        torch.empty((batch, r, returns), dtype=torch.int64, device=device),
        torch.empty((batch, r, returns), dtype=torch.bool, device=device),
        torch.empty((batch, r, returns), dtype=torch.int64, device=device),
        torch.empty((batch, r), dtype=torch.int32, device=device),
    ]
    mod.render_lidar(descriptors, len(case["scenes"]), inputs, outputs, counters, returns, packet,
                     defaults.near_plane_m, defaults.far_plane_m, defaults.support_sigma,
                     defaults.detection_threshold, defaults.planarity_ratio_max, defaults.min_incidence_cos,
                     defaults.cluster_abs_m, defaults.cluster_relative, defaults.fallback_reflectivity,
                     defaults.direction_norm_tolerance, defaults.semantic_slots)
    torch.cuda.synchronize()
    names = ("range_m", "position_world_m", "intensity", "semantic_id", "valid", "time_offset_ns", "return_count")
    return {n: t.cpu().numpy() for n, t in zip(names, outputs)}, counters.cpu().tolist()


@pytest.mark.parametrize("name", lidar_cases.names())
@pytest.mark.parametrize("packet", [8, 16])
def test_lidar_native_module_matches_reference_golden(name, packet):
    case = lidar_cases.load(name)
    got, counters = _render_through_module(case, packet)
    want = case["expected"]
    for key in ("valid", "semantic_id", "return_count", "time_offset_ns"):
        np.testing.assert_array_equal(got[key], np.asarray(want[key]).astype(got[key].dtype), err_msg=key)
    valid = np.asarray(want["valid"]).astype(bool)
    np.testing.assert_allclose(got["range_m"][valid], want["range_m"][valid], rtol=0, atol=1e-4)
    np.testing.assert_allclose(got["intensity"][valid], want["intensity"][valid], rtol=0, atol=1e-4)
    assert np.all(np.isinf(got["range_m"][~valid]))
    assert counters[6] == int(valid.sum())  # returns
    assert counters[0] == counters[1] == 1  # calls started / completed


def test_lidar_native_module_contract_errors():
    mod = load_lidar_extension()
    device = torch.device("cuda")
    with pytest.raises(RuntimeError, match="num_items must be positive"):
        mod.sort_temp_bytes(0)
    means = torch.zeros((16, 3), device=device)
    with pytest.raises(RuntimeError, match="packet_size must be 8 or 16"):
        mod.build_scene_lbvh([means, means, torch.zeros((16, 4), device=device)], [means] * 7, 4, 2, 2, 3.0, 0.35)
    descriptors = torch.zeros((2, 14), dtype=torch.int64, device=device)
    scene = [means, means, torch.zeros((16, 4), device=device), torch.zeros(16, device=device),
             torch.zeros(16, dtype=torch.int64, device=device), means, means, means,
             torch.zeros((3, 6), device=device)]
    with pytest.raises(RuntimeError, match="needs build_scene_lbvh"):
        mod.pack_scene_descriptor(descriptors, 0, 1, scene, 2, 2)
