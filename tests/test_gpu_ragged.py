"""Ragged batched form vs the CPU oracle: cameras of different resolutions
over scenes of different sizes in one submission.

Every camera of the ragged rig is rendered by the oracle on its own (at its
own resolution, with its own scene) and compared bit for bit with its view
of the flat outputs, together with its tiles' sorted Gaussian lists; the
frame counters are the sums over cameras.  The ragged frame is also
repeated, and captured in a CUDA graph and replayed with new poses.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from helpers import assert_bitwise_equal, render_oracle
from vgr_b200 import CustomCudaBackend, RendererService
from vgr_b200.ragged import RaggedBatch, autotune_tile_size
from vgr_b200.workloads import CameraRig, look_at_viewmats, pinhole, synthetic_scene

pytestmark = pytest.mark.gpu

RESOLUTIONS = [(64, 48), (96, 72), (40, 56), (128, 128), (33, 17), (64, 48), (120, 160)]
SCENE_IDS = [3, 8, 3, 8, 99, 3, 8]  # 99 is unregistered: the camera stays background


def _scenes():
    return [
        (3, synthetic_scene(6_000, seed=81, mean_half_extent=1.2, log_scale_mean=-3.4, sh_degree=2)),
        (8, synthetic_scene(15_000, seed=82, mean_half_extent=1.6, log_scale_mean=-3.8, sh_degree=2)),
    ]


def _poses(seed: int):
    gen = torch.Generator().manual_seed(seed)
    count = len(RESOLUTIONS)
    angle = torch.rand((count,), generator=gen, dtype=torch.float64) * 6.283
    eyes = torch.stack((3.5 * torch.cos(angle), 0.6 + 0.4 * torch.rand((count,), generator=gen, dtype=torch.float64),
                        3.5 * torch.sin(angle)), dim=1)
    view = look_at_viewmats(eyes, torch.zeros((count, 3), dtype=torch.float64))
    intr = torch.zeros((count, 3, 3))
    for c, (h, w) in enumerate(RESOLUTIONS):
        intr[c] = pinhole(1, 0.9 * w, 0.9 * w, w / 2.0, h / 2.0)[0]
    return view, intr


def _setup(tile_size, persistent_compositor=False, composite_shape=0):
    device = torch.device("cuda")
    # The backend keeps the reference's tile contract (<= 16); the ragged
    # form takes its own tile size (32-pixel tiles included).
    backend = CustomCudaBackend(sh_degree=2, output_srgb=False, tile_size=min(tile_size, 16))
    service = RendererService(backend, height=64, width=64, max_views=1)
    service.initialize(stage=None, device=device)
    for sid, scene in _scenes():
        service.load_scene(sid, **scene.to(device).as_kwargs())
    heights = [h for h, _ in RESOLUTIONS]
    widths = [w for _, w in RESOLUTIONS]
    return RaggedBatch(backend, heights, widths, tile_size=tile_size,
                       persistent_compositor=persistent_compositor, composite_shape=composite_shape), device


def _check_against_oracle(ragged, outputs, view, intr, tile_size):
    ws = ragged.workspace
    starts = ws["tile_starts"].cpu().numpy()
    ends = ws["tile_ends"].cpu().numpy()
    values = ws["values_out"].cpu().numpy()
    gids = ws["records"].view(torch.int32)[:, 7].cpu().numpy()
    tile_offsets = ragged._tile_offsets_t.cpu().numpy()
    visible = intersections = 0
    for c, (h, w) in enumerate(RESOLUTIONS):
        rig = CameraRig(view[c:c + 1].contiguous(), intr[c:c + 1].contiguous(), h, w)
        cpu = render_oracle(_scenes(), rig, [SCENE_IDS[c]], tile_size=tile_size, sh_degree=2, with_tiles=True)
        visible += cpu.visible
        intersections += cpu.intersections
        for name, want in (("rgb", cpu.rgb), ("depth", cpu.depth), ("alpha", cpu.alpha),
                           ("semantic_id", cpu.semantic)):
            got = ragged.view(outputs, name, c).cpu().numpy()
            assert_bitwise_equal(got, want[0], f"camera {c} {name}")
        t0, t1 = tile_offsets[c], tile_offsets[c + 1]
        counts = (ends[t0:t1] - starts[t0:t1]).astype(np.int32)
        assert_bitwise_equal(counts, cpu.tile_counts, f"camera {c} tile counts")
        ids = np.concatenate([gids[values[starts[t]:ends[t]]] for t in range(t0, t1)] + [np.zeros(0, np.int32)])
        assert_bitwise_equal(ids.astype(np.int32), cpu.sorted_gaussian_ids.astype(np.int32), f"camera {c} sorted ids")
    counters = ragged.check()
    assert counters["visible_gaussians"] == visible
    assert counters["tile_intersections"] == intersections


# Every autotuner candidate: tile size x compositor launch x CTA shape
# (composite_shape 0 two pixels per thread, 1 one pixel per thread, 2 two
# pixels per thread at half occupancy) renders the oracle's bits.
@pytest.mark.parametrize(
    "tile_size,persistent,shape",
    [(8, False, 0), (8, False, 1), (8, True, 1), (8, False, 2), (8, True, 2), (16, False, 0), (16, True, 0),
     (16, False, 1), (16, True, 1), (16, False, 2), (16, True, 2), (32, False, 0), (32, True, 0), (32, False, 1),
     (32, False, 2), (32, True, 2)],
)
def test_ragged_batch_matches_oracle_per_camera(tile_size, persistent, shape):
    ragged, device = _setup(tile_size, persistent, shape)
    view, intr = _poses(1)
    vm, km = view.to(device), intr.to(device)
    ids = torch.tensor(SCENE_IDS, dtype=torch.int64, device=device)
    outputs = ragged.outputs()
    ragged.calibrate(vm, km, ids, outputs)
    _check_against_oracle(ragged, outputs, view, intr, tile_size)
    first = {k: v.clone() for k, v in outputs.items()}
    ragged.render(vm, km, ids, outputs)
    torch.cuda.synchronize()
    for name in first:
        assert torch.equal(first[name], outputs[name]), name


def test_ragged_graph_replay_with_new_poses():
    ragged, device = _setup(16)
    view, intr = _poses(2)
    vm, km = view.to(device), intr.to(device)
    ids = torch.tensor(SCENE_IDS, dtype=torch.int64, device=device)
    outputs = ragged.outputs()
    ragged.calibrate(vm, km, ids, outputs)
    graph = ragged.capture(vm, km, ids, outputs)
    view2, _ = _poses(3)
    vm.copy_(view2.to(device))
    graph.replay()
    torch.cuda.synchronize()
    replayed = {k: v.clone() for k, v in outputs.items()}
    ragged.render(vm, km, ids, outputs)
    torch.cuda.synchronize()
    for name in replayed:
        assert torch.equal(replayed[name], outputs[name]), name
    _check_against_oracle(ragged, outputs, view2, intr, 16)


def test_autotuner_picks_a_candidate_and_caches_it():
    ragged, device = _setup(16)
    view, intr = _poses(4)
    vm, km = view.to(device), intr.to(device)
    ids = torch.tensor(SCENE_IDS, dtype=torch.int64, device=device)
    outputs = ragged.outputs()
    cache = {}
    kw = {"candidates": (8, 16, 32), "persistent_candidates": (False, True), "shape_candidates": (0, 1, 2),
          "cache": cache}
    tile = autotune_tile_size(ragged, vm, km, ids, outputs, **kw)
    persistent, shape = ragged.persistent_compositor, ragged.composite_shape
    assert tile in (8, 16, 32) and ragged.tile_size == tile and len(cache) == 1
    # Tiles 8 (shapes 0, 1), 16 and 32 (shapes 0, 1, 2), each with both launches.
    assert len(ragged.autotune_ms) == 16
    assert autotune_tile_size(ragged, vm, km, ids, outputs, **kw) == tile
    assert (ragged.persistent_compositor, ragged.composite_shape) == (persistent, shape) and len(cache) == 1
    ragged.render(vm, km, ids, outputs)
    _check_against_oracle(ragged, outputs, view, intr, tile)
