"""CUDA camera path vs the CPU oracle on identical seeded inputs.

The kernels and the oracle execute the same IEEE operation sequence, so the
comparison is bit-exact for every output (RGB, alpha, depth, semantic),
for the frame counters and for the per-tile sorted Gaussian lists -- a
stricter bar than the 1e-4 float tolerance stated for the path.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from helpers import assert_bitwise_equal, render_gpu, render_oracle
from vgr_b200.workloads import (
    CameraRig,
    look_at_viewmats,
    orbit_cameras,
    pinhole,
    plain_workload,
    synthetic_scene,
)

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


def _small_rig(batch=4, width=96, height=80, seed=3, radius=4.0):
    rig = orbit_cameras(batch, seed=seed, radius=radius, height_offset=0.8, width=width, height=height, focal=90.0)
    return rig


def test_plain_config_bitwise():
    scene, rig = plain_workload()
    gpu = render_gpu([(0, scene)], rig, [0])
    cpu = render_oracle([(0, scene)], rig, [0], with_tiles=True)
    _compare(gpu, cpu)
    assert_bitwise_equal(_sorted_gids(gpu), cpu.sorted_gaussian_ids, "sorted gaussian ids")
    starts = gpu.backend.workspace["tile_starts"].cpu().numpy()
    ends = gpu.backend.workspace["tile_ends"].cpu().numpy()
    assert_bitwise_equal((ends - starts).astype(np.int32), cpu.tile_counts, "per-tile counts")


@pytest.mark.parametrize("tile_size,shape", [(4, 0), (8, 0), (8, 1), (16, 0), (16, 1), (16, 2)])
def test_batched_tile_sizes_bitwise(tile_size, shape):
    scene = synthetic_scene(20_000, seed=5, mean_half_extent=1.5, log_scale_mean=-3.5)
    rig = _small_rig()
    gpu = render_gpu([(7, scene)], rig, [7] * 4, tile_size=tile_size, composite_shape=shape)
    cpu = render_oracle([(7, scene)], rig, [7] * 4, tile_size=tile_size, with_tiles=True)
    _compare(gpu, cpu)
    assert_bitwise_equal(_sorted_gids(gpu), cpu.sorted_gaussian_ids, "sorted gaussian ids")


def test_multi_scene_active_subset_bitwise():
    scenes = [
        (11, synthetic_scene(3_000, seed=11, mean_half_extent=1.0)),
        (12, synthetic_scene(17_000, seed=12, mean_half_extent=1.2, log_scale_mean=-3.2)),
        (13, synthetic_scene(500, seed=13, mean_half_extent=0.5, log_scale_mean=-2.5)),
    ]
    rig = _small_rig(batch=6, width=72, height=56, seed=9, radius=3.5)
    scene_ids = [12, 11, 13, 12, 99, 11]  # 99 is unregistered: background
    active = [5, 0, 2, 4, 1, 17]  # 17 is outside the batch: skipped
    gpu = render_gpu(scenes, rig, scene_ids, active_ids=active)
    cpu = render_oracle(scenes, rig, scene_ids, active_ids=active)
    # Inactive cameras (3) keep the reset contract; active ones match the oracle.
    inactive = 3
    out = gpu.outputs
    assert torch.all(out["rgb"][inactive] == 0)
    assert torch.all(torch.isinf(out["depth"][inactive]))
    assert torch.all(out["semantic_id"][inactive] == -1)
    for cam in (0, 1, 2, 4, 5):
        assert_bitwise_equal(out["rgb"][cam].cpu().numpy(), cpu.rgb[cam], f"rgb[{cam}]")
        assert_bitwise_equal(out["depth"][cam].cpu().numpy(), cpu.depth[cam], f"depth[{cam}]")
        assert_bitwise_equal(out["alpha"][cam].cpu().numpy(), cpu.alpha[cam], f"alpha[{cam}]")
        assert_bitwise_equal(out["semantic_id"][cam].cpu().numpy(), cpu.semantic[cam], f"semantic[{cam}]")
    assert gpu.counters["visible_gaussians"] == cpu.visible
    assert gpu.counters["tile_intersections"] == cpu.intersections


def test_sh3_antialiased_srgb_bitwise():
    scene = synthetic_scene(15_000, seed=21, mean_half_extent=1.5, log_scale_mean=-3.4, sh_degree=3)
    rig = _small_rig(batch=3, width=64, height=64, seed=4)
    kwargs = dict(sh_degree=3, rasterize_mode="antialiased", output_srgb=True)
    gpu = render_gpu([(1, scene)], rig, [1, 1, 1], **kwargs)
    cpu = render_oracle([(1, scene)], rig, [1, 1, 1], **kwargs)
    _compare(gpu, cpu)


def test_rgb_only_contract_bitwise():
    scene = synthetic_scene(8_000, seed=31, mean_half_extent=1.0)
    rig = _small_rig(batch=2, width=48, height=40, seed=6, radius=3.0)
    gpu = render_gpu([(2, scene)], rig, [2, 2], outputs=("rgb",))
    cpu = render_oracle([(2, scene)], rig, [2, 2])
    assert_bitwise_equal(gpu.outputs["rgb"].cpu().numpy(), cpu.rgb, "rgb")


def test_capacity_growth_matches_oracle():
    scene = synthetic_scene(20_000, seed=41, mean_half_extent=1.5, log_scale_mean=-3.0)
    rig = _small_rig(batch=2, seed=8)
    gpu = render_gpu([(3, scene)], rig, [3, 3], max_visible_records=64, max_intersections=128)
    cpu = render_oracle([(3, scene)], rig, [3, 3])
    _compare(gpu, cpu)
    stats = gpu.backend.capacity_stats
    assert stats["totals"]["growth_events"] >= 1
    assert stats["last_render"]["status"] == "success"


def test_repeat_is_bitwise_stable_and_equal_depth_ties_follow_gaussian_id():
    # Layout of the reference's deterministic smoke: identical Gaussians at
    # one depth; within a tile they must be ordered by Gaussian id and the
    # centre semantic is the lowest id (strict > keeps the earliest weight).
    count = 256
    scene = synthetic_scene(count, seed=0)
    scene.means.zero_()
    scene.means[:, 2] = 5.0
    scene.scales.fill_(0.03)
    scene.rotations.zero_()
    scene.rotations[:, 0] = 1.0
    scene.opacities.fill_(0.2)
    scene.features.zero_()
    scene.features[:, 0] = torch.linspace(1.0, 0.0, count)
    scene.semantic_ids.copy_(torch.arange(1000, 1000 + count))
    view = torch.eye(4).repeat(2, 1, 1)
    view[:, 2, 3] = -4.0
    rig = CameraRig(view.contiguous(), pinhole(2, 64.0, 64.0, 32.0, 32.0), 64, 64)
    gpu = render_gpu([(73, scene)], rig, [73, 73], gaussian_support_sigma=3.0, deterministic=True)
    first = {k: v.clone() for k, v in gpu.outputs.items()}
    for _ in range(3):
        gpu.service.render(
            rig.viewmats.cuda(), rig.intrinsics.cuda(), torch.tensor([73, 73], device="cuda"),
            outputs=gpu.outputs,
        )
    gpu.service.synchronize()
    for name in first:
        assert torch.equal(first[name], gpu.outputs[name]), name
    ws = gpu.backend.workspace
    tile = (32 // 16) * 4 + (32 // 16)
    start, end = int(ws["tile_starts"][tile]), int(ws["tile_ends"][tile])
    gids = ws["records"].view(torch.int32)[:, 7][ws["values_out"][start:end].long()]
    assert torch.equal(gids.cpu(), torch.arange(count, dtype=torch.int32))
    assert int(gpu.outputs["semantic_id"][0, 32, 32, 0]) == 1000
    cpu = render_oracle([(73, scene)], rig, [73, 73], gaussian_support_sigma=3.0)
    _compare(gpu, cpu)


def test_everything_culled_and_empty_tiles():
    scene = synthetic_scene(1_000, seed=51)
    eyes = torch.tensor([[0.0, 0.0, 10.0]])
    view = look_at_viewmats(eyes, torch.tensor([[0.0, 0.0, 20.0]]))  # looking away
    rig = CameraRig(view, pinhole(1, 50.0, 50.0, 16.0, 16.0), 32, 32)
    gpu = render_gpu([(0, scene)], rig, [0])
    assert gpu.counters["visible_gaussians"] == 0
    assert gpu.counters["tile_intersections"] == 0
    assert torch.all(gpu.outputs["rgb"] == 0)
    assert torch.all(gpu.outputs["alpha"] == 0)
    assert torch.all(torch.isinf(gpu.outputs["depth"]))
    assert torch.all(gpu.outputs["semantic_id"] == -1)


def _dense_cluster_rig():
    eyes = torch.tensor([[0.0, 0.0, -3.0]])
    view = look_at_viewmats(eyes, torch.zeros((1, 3)))
    return CameraRig(view, pinhole(1, 256.0, 256.0, 64.0, 64.0), 128, 128)


def test_buckets_above_shared_memory_capacity_bitwise():
    # A tight cluster puts tens of thousands of keys into a handful of tiles,
    # which the tile sort orders in chunks through global memory.
    scene = synthetic_scene(30_000, seed=61, mean_half_extent=0.04, log_scale_mean=-5.0)
    rig = _dense_cluster_rig()
    gpu = render_gpu([(0, scene)], rig, [0])
    cpu = render_oracle([(0, scene)], rig, [0], with_tiles=True)
    assert cpu.tile_counts.max() > 4096
    _compare(gpu, cpu)
    assert_bitwise_equal(_sorted_gids(gpu), cpu.sorted_gaussian_ids, "sorted gaussian ids")


def test_large_bucket_of_equal_depths_follows_gaussian_id():
    count = 6_000
    scene = synthetic_scene(count, seed=62, log_scale_mean=-5.5)
    scene.means[:, :2] = (torch.rand((count, 2), generator=torch.Generator().manual_seed(3)) - 0.5) * 0.02
    scene.means[:, 2] = 0.0
    rig = _dense_cluster_rig()
    gpu = render_gpu([(0, scene)], rig, [0])
    cpu = render_oracle([(0, scene)], rig, [0], with_tiles=True)
    assert cpu.tile_counts.max() > 4096
    _compare(gpu, cpu)
    assert_bitwise_equal(_sorted_gids(gpu), cpu.sorted_gaussian_ids, "sorted gaussian ids")


def test_partial_depth_ties_in_shared_memory_buckets():
    # Half of the Gaussians share one of three depths, the rest are spread:
    # buckets below the shared-memory capacity take the tie re-sort.
    count = 3_000
    scene = synthetic_scene(count, seed=63, mean_half_extent=0.05, log_scale_mean=-5.0)
    scene.means[::2, 2] = torch.tensor([-0.01, 0.0, 0.01]).repeat(count // 6 + 1)[: (count + 1) // 2]
    rig = _dense_cluster_rig()
    gpu = render_gpu([(0, scene)], rig, [0])
    cpu = render_oracle([(0, scene)], rig, [0], with_tiles=True)
    assert 1 < cpu.tile_counts.max() <= 4096
    _compare(gpu, cpu)
    assert_bitwise_equal(_sorted_gids(gpu), cpu.sorted_gaussian_ids, "sorted gaussian ids")


@pytest.mark.parametrize("count", [2_400, 16_000])
def test_paired_depth_ties_in_radix_sorted_buckets(count):
    # Most Gaussians sit in a thin depth band (splits above the insertion-sort
    # limit, so buckets take the radix passes) and come in pairs at the same
    # position: short runs of equal depth inside radix-sorted buckets, below
    # (2,400) and above (16,000) the shared-memory capacity.
    scene = synthetic_scene(count, seed=64, mean_half_extent=0.05, log_scale_mean=-5.0)
    gen = torch.Generator().manual_seed(5)
    band = torch.arange(count // 2, dtype=torch.float32) * 1e-6
    spread = (torch.rand((count // 2,), generator=gen) - 0.5) * 0.04
    z = torch.where(torch.arange(count // 2) % 5 == 0, spread, band)
    scene.means[0::2, 2] = z
    scene.means[1::2] = scene.means[0::2]
    rig = _dense_cluster_rig()
    gpu = render_gpu([(0, scene)], rig, [0])
    cpu = render_oracle([(0, scene)], rig, [0], with_tiles=True)
    if count > 6_000:
        assert cpu.tile_counts.max() > 4096
    else:
        assert 1 < cpu.tile_counts.max() <= 3072
    _compare(gpu, cpu)
    assert_bitwise_equal(_sorted_gids(gpu), cpu.sorted_gaussian_ids, "sorted gaussian ids")


def test_large_tile_grid_bitwise():
    # 19,200 4x4-pixel tiles over four 320x240 cameras.
    scene = synthetic_scene(20_000, seed=71, mean_half_extent=1.5, log_scale_mean=-3.5)
    rig = orbit_cameras(4, seed=12, radius=4.0, height_offset=0.8, width=320, height=240, focal=260.0)
    gpu = render_gpu([(2, scene)], rig, [2] * 4, tile_size=4)
    cpu = render_oracle([(2, scene)], rig, [2] * 4, tile_size=4, with_tiles=True)
    assert cpu.tile_counts.size >= 4096
    _compare(gpu, cpu)
    assert_bitwise_equal(_sorted_gids(gpu), cpu.sorted_gaussian_ids, "sorted gaussian ids")


def _check_cluster_bounds(packed) -> None:
    # Each cluster row bounds its 32 Gaussians' means and holds their largest
    # covariance trace; clusters past a scene's end hold an empty box.
    means = packed["means"].cpu().numpy()
    cov = packed["covariances"].cpu().numpy()
    offsets = packed["scene_offsets"].cpu().tolist()
    chunk_offsets = packed["chunk_offsets"].cpu().tolist()
    rows = packed["cluster_bounds"].cpu().numpy()
    for s in range(len(offsets) - 1):
        count = offsets[s + 1] - offsets[s]
        for k in range(-(-count // 512) * 16):
            row = rows[chunk_offsets[s] * 16 + k]
            g0, g1 = offsets[s] + 32 * k, min(offsets[s] + 32 * k + 32, offsets[s + 1])
            if g0 >= offsets[s + 1]:
                assert np.all(row[:3] == np.inf) and np.all(row[4:7] == -np.inf), (s, k, row)
                continue
            m = means[g0:g1]
            np.testing.assert_array_equal(row[:3], m.min(axis=0))
            np.testing.assert_array_equal(row[4:7], m.max(axis=0))
            trace = cov[g0:g1, 0] + cov[g0:g1, 3] + cov[g0:g1, 5]
            assert row[3] == trace.astype(np.float32).max(), (s, k)


def test_spatial_layout_renders_identically():
    # Scenes stored in Morton order with per-chunk frustum culling render
    # exactly what the scene in id order renders: cameras inside a large
    # scene (so most chunks are outside each frustum), two scenes, ties by id.
    scenes = [
        (4, synthetic_scene(40_000, seed=91, mean_half_extent=6.0, log_scale_mean=-3.0, sh_degree=1)),
        (6, synthetic_scene(9_000, seed=92, mean_half_extent=2.0, log_scale_mean=-3.5, sh_degree=1)),
    ]
    eyes = torch.tensor([[0.0, 0.5, 0.0], [3.0, 0.0, -2.0], [0.0, 0.0, 4.0], [0.5, 1.0, 0.5]])
    targets = torch.tensor([[5.0, 0.0, 0.0], [3.0, 0.0, 5.0], [0.0, 0.0, 0.0], [-4.0, 0.0, 0.0]])
    rig = CameraRig(look_at_viewmats(eyes, targets), pinhole(4, 70.0, 70.0, 48.0, 32.0), 64, 96)
    ids = [4, 4, 6, 4]
    with_layout = render_gpu(scenes, rig, ids, sh_degree=1, spatial_layout=True)
    without = render_gpu(scenes, rig, ids, sh_degree=1, spatial_layout=False)
    packed = with_layout.backend._packed_scene
    assert "chunk_bounds" in packed and "cluster_bounds" in packed
    _check_cluster_bounds(packed)
    for name in ("rgb", "depth", "alpha", "semantic_id"):
        assert torch.equal(with_layout.outputs[name], without.outputs[name]), name
    assert with_layout.counters == without.counters
    assert_bitwise_equal(_sorted_gids(with_layout), _sorted_gids(without), "sorted gaussian ids")
    cpu = render_oracle(scenes, rig, ids, sh_degree=1)
    _compare(with_layout, cpu)
