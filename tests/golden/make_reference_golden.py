"""Generate camera golden vectors by running the reference's own CUDA build.

Runs on a CUDA machine with oracle/_ref/vgr_reference_camera.so built by
oracle/build_ref.py from the reference sources
(src/isaacsim_gaussian_renderer/native/renderer.cpp + renderer_cuda.cu, its
own flags -O3 --use_fast_math).  For each seeded synthetic case it calls the
reference extension's ``render`` with a workspace laid out like the
reference backend's plan (cuda_backend.py:1021-1327, tile path, no dense
1x1 buffers) and stores the outputs, counters, per-tile intersection counts
and the per-tile sorted Gaussian ids in tests/golden/camera_<case>.npz.
The inputs are regenerated from the seeds by the tests, so only outputs are
stored.

Usage: python tests/golden/make_reference_golden.py [--out DIR]
"""

from __future__ import annotations

import argparse
import sys
from pathlib import Path

import numpy as np
import torch

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT / "vectorized-gaussian-renderer-public_b200"))
sys.path.insert(0, str(ROOT))

from oracle.build_ref import load_reference_module  # noqa: E402
from tests.golden.cases import CASES  # noqa: E402


def render_reference(ref, case, device):
    scenes, rig, scene_ids = case["build"]()
    opts = case["options"]
    means = torch.cat([s.means for _, s in scenes]).to(device).contiguous()
    scales = torch.cat([s.scales for _, s in scenes]).to(device).contiguous()
    rotations = torch.cat([s.rotations for _, s in scenes]).to(device).contiguous()
    opacities = torch.cat([s.opacities for _, s in scenes]).to(device).contiguous()
    features = torch.cat([s.features for _, s in scenes]).to(device).contiguous()
    semantic = torch.cat([s.semantic_ids for _, s in scenes]).to(device).contiguous()
    covariances = torch.empty((means.shape[0], 6), device=device)
    ref.precompute_covariances(scales, rotations, covariances)
    counts = [s.means.shape[0] for _, s in scenes]
    offsets = torch.tensor(np.cumsum([0] + counts), dtype=torch.int64, device=device)
    registered = torch.tensor([sid for sid, _ in scenes], dtype=torch.int64, device=device)
    batch = rig.viewmats.shape[0]
    h, w = rig.height, rig.width
    ts = opts.get("tile_size", 16)
    ray = opts.get("ray_gaussian_evaluation", False)
    bin_size = 32 if ray and ts == 16 else ts  # renderer_cuda.cu:2670-2676
    tiles = batch * (-(-h // bin_size)) * (-(-w // bin_size))
    visible_cap = batch * sum(counts)
    isect_cap = max(visible_cap * 64, 1024)
    deterministic = opts.get("deterministic", True)
    f32, i32, i64 = torch.float32, torch.int32, torch.int64
    temp_bytes = (
        ref.sort_temp_bytes(isect_cap, tiles)
        if deterministic
        else ref.radix_sort_double_buffer_temp_bytes(isect_cap, tiles)
    )
    ws = [
        torch.zeros((visible_cap, 2), dtype=f32, device=device),
        torch.zeros((visible_cap, 3), dtype=f32, device=device),
        torch.zeros((visible_cap,), dtype=f32, device=device),
        torch.zeros((visible_cap,), dtype=f32, device=device),
        torch.zeros((visible_cap,), dtype=i32, device=device),
        torch.zeros((visible_cap,), dtype=i32, device=device),
        torch.zeros((visible_cap, 2), dtype=i32, device=device),
        torch.zeros((isect_cap,), dtype=torch.uint64, device=device),
        torch.zeros((isect_cap,), dtype=torch.uint64, device=device),
        torch.zeros((isect_cap,), dtype=i32, device=device),
        torch.zeros((isect_cap,), dtype=i32, device=device),
        torch.zeros((tiles,), dtype=i32, device=device),
        torch.zeros((tiles,), dtype=i32, device=device),
        torch.zeros((5,), dtype=i64, device=device),
        torch.zeros((max(temp_bytes, 1),), dtype=torch.uint8, device=device),
        torch.zeros((1, 1), dtype=f32, device=device),
        torch.zeros((1,), dtype=i32, device=device),
        torch.zeros((1,), dtype=i64, device=device),
        torch.zeros((1,), dtype=i64, device=device),
        torch.zeros((1,), dtype=i64, device=device),
        torch.zeros((1,), dtype=i32, device=device),
        torch.zeros((1,), dtype=f32, device=device),
        torch.zeros((visible_cap if ray else 1, 6), dtype=f32, device=device),
        torch.zeros((visible_cap if ray else 1, 4), dtype=f32, device=device),
    ]
    out = [
        torch.zeros((batch, h, w, 3), dtype=f32, device=device),
        torch.zeros((batch, h, w, 1), dtype=f32, device=device),
        torch.zeros((batch, h, w, 1), dtype=f32, device=device),
        torch.zeros((batch, h, w, 1), dtype=i64, device=device),
    ]
    cams = [
        rig.viewmats.to(device).contiguous(),
        rig.intrinsics.to(device).contiguous(),
        torch.eye(4, device=device).repeat(batch, 1, 1).contiguous(),
        torch.tensor(scene_ids, dtype=i64, device=device),
        torch.empty((0,), dtype=i64, device=device),
    ]
    selector = ref.render(
        [means, covariances, opacities, features, semantic, registered, offsets],
        cams,
        out,
        ws,
        h,
        w,
        max(counts),
        opts.get("near_plane", 0.01),
        opts.get("far_plane", 100.0),
        opts.get("gaussian_support_sigma", 3.33),
        opts.get("covariance_epsilon", 0.3),
        opts.get("rasterize_mode", "classic") == "antialiased",
        opts.get("semantic_min_alpha", 0.01),
        ray,
        ts,
        4096,
        64,
        False,
        False,
        False,
        opts.get("output_srgb", False),
        deterministic,
        True,
        False,
    )
    torch.cuda.synchronize()
    counters = ws[13].cpu().numpy()
    n = int(min(counters[1], isect_cap))
    values = (ws[10] if selector == 1 else ws[9])[:n].long()
    sorted_gids = ws[5][values].cpu().numpy()
    tile_counts = (ws[12] - ws[11]).cpu().numpy()
    return {
        "rgb": out[0].cpu().numpy(),
        "depth": out[1].cpu().numpy(),
        "alpha": out[2].cpu().numpy(),
        "semantic": out[3].cpu().numpy(),
        "counters": counters,
        "tile_counts": tile_counts,
        "sorted_gaussian_ids": sorted_gids.astype(np.int32),
        "selector": np.int64(selector),
    }


def main() -> None:
    parser = argparse.ArgumentParser()
    parser.add_argument("--out", type=Path, default=Path(__file__).resolve().parent)
    parser.add_argument("--cases", nargs="*", default=None, help="subset of case names")
    args = parser.parse_args()
    device = torch.device("cuda")
    ref = load_reference_module("vgr_reference_camera")
    args.out.mkdir(parents=True, exist_ok=True)
    for name, case in CASES.items():
        if args.cases and name not in args.cases:
            continue
        result = render_reference(ref, case, device)
        path = args.out / f"camera_{name}.npz"
        np.savez_compressed(path, **result)
        print(name, {k: (v.shape if hasattr(v, "shape") else v) for k, v in result.items()},
              "counters", result["counters"].tolist())


if __name__ == "__main__":
    main()
