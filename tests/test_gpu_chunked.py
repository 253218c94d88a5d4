"""Logical -> physical chunked submission (cuda_backend.py:759-967,
renderer_cuda.cu:2307-2360) vs the CPU oracle.

A logical batch of five cameras renders as physical submissions of two
cameras with fixed-capacity sorting and no host read; with an active subset
the device maps logical active ids to per-chunk ids
(``prepare_chunked_active_ids``) and the chunk counters are summed on the
device (``aggregate_chunk_counters``).  Outputs are bit-identical to the
oracle's single render of the whole batch.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from helpers import assert_bitwise_equal, render_oracle
from vgr_b200 import CustomCudaBackend, RendererService
from vgr_b200.workloads import orbit_cameras, synthetic_scene

pytestmark = pytest.mark.gpu


def _service():
    device = torch.device("cuda")
    scene = synthetic_scene(15_000, seed=61, mean_half_extent=1.5, log_scale_mean=-3.5)
    rig = orbit_cameras(5, seed=9, radius=4.0, height_offset=0.6, width=80, height=64, focal=75.0)
    backend = CustomCudaBackend(output_srgb=False, max_physical_views=2, fixed_capacity_sort=True,
                                deterministic=False, adaptive_capacity=False)
    service = RendererService(backend, height=rig.height, width=rig.width, max_views=5)
    service.initialize(stage=None, device=device)
    service.load_scene(3, **scene.to(device).as_kwargs())
    backend.reserve_workspace_capacity(visible_records=2 * 15_000, tile_intersections=400_000)
    return scene, rig, backend, service, device


def test_chunked_logical_batch_matches_oracle():
    scene, rig, backend, service, device = _service()
    out = service.render(rig.viewmats.to(device), rig.intrinsics.to(device),
                         torch.full((5,), 3, dtype=torch.int64, device=device))
    service.synchronize()
    cpu = render_oracle([(3, scene)], rig, [3] * 5)
    for name, want in (("rgb", cpu.rgb), ("depth", cpu.depth), ("alpha", cpu.alpha), ("semantic_id", cpu.semantic)):
        assert_bitwise_equal(out[name].cpu().numpy(), want, name)
    counters = backend.read_counters()
    assert counters["visible_gaussians"] == cpu.visible
    assert counters["tile_intersections"] == cpu.intersections
    assert counters["visible_overflow"] == 0 and counters["intersection_overflow"] == 0


def test_chunked_active_subset_matches_oracle():
    scene, rig, backend, service, device = _service()
    active = [4, 1, 3]
    out = service.render(rig.viewmats.to(device), rig.intrinsics.to(device),
                         torch.full((5,), 3, dtype=torch.int64, device=device),
                         active_camera_ids=torch.tensor(active, dtype=torch.int64, device=device))
    service.synchronize()
    cpu = render_oracle([(3, scene)], rig, [3] * 5, active_ids=active)
    for cam in active:
        for name, want in (("rgb", cpu.rgb), ("depth", cpu.depth), ("alpha", cpu.alpha),
                           ("semantic_id", cpu.semantic)):
            assert_bitwise_equal(out[name][cam].cpu().numpy(), want[cam], f"camera {cam} {name}")
    counters = backend.read_counters()
    assert counters["visible_gaussians"] == cpu.visible
    assert counters["tile_intersections"] == cpu.intersections
    assert np.isfinite(out["rgb"][[4, 1, 3]].cpu().numpy()).all()
