"""Time the reference's own CUDA camera path beside this build's on one GPU.

Test infrastructure, not part of the product: it runs the reference
extension compiled from its sources (oracle/_ref/vgr_reference_camera.so,
built by oracle/build_ref.py) on the batched workload (1M Gaussians, 64
cameras 640x480) with linear-RGB features (the reference reads features[0..2]
as RGB), and this build's CustomCudaBackend on the same inputs with the same
equation (sh_degree=None), through RendererService.  Both are timed with CUDA
events over K frames after warm-up; the reference in its deterministic
(segmented-sort) and global-radix modes.  The outputs of the two are compared
as a parity check at full size.

Usage: python tests/golden/time_reference_cuda.py [--frames 10] [--out gpurun_out/ref_cuda.json]
"""

from __future__ import annotations

import argparse
import json
import sys
from pathlib import Path

import numpy as np
import torch

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT / "vectorized-gaussian-renderer-public_b200"))
sys.path.insert(0, str(ROOT))

from oracle.build_ref import load_reference_module  # noqa: E402
from vgr_b200 import CustomCudaBackend, RendererService  # noqa: E402
from vgr_b200.workloads import batched_workload  # noqa: E402


def reference_frame(ref, scene, rig, device, deterministic: bool, frames: int):
    f32, i32, i64 = torch.float32, torch.int32, torch.int64
    means, scales, rotations = (t.to(device).contiguous() for t in (scene.means, scene.scales, scene.rotations))
    opacities, features = scene.opacities.to(device).contiguous(), scene.features.to(device).contiguous()
    semantic = scene.semantic_ids.to(device).contiguous()
    covariances = torch.empty((means.shape[0], 6), device=device)
    ref.precompute_covariances(scales, rotations, covariances)
    g = means.shape[0]
    batch, h, w, ts = rig.viewmats.shape[0], rig.height, rig.width, 16
    tiles = batch * (-(-h // ts)) * (-(-w // ts))
    visible_cap, isect_cap = batch * g, 160_000_000
    temp_bytes = (ref.sort_temp_bytes(isect_cap, tiles) if deterministic
                  else ref.radix_sort_double_buffer_temp_bytes(isect_cap, tiles))
    ws = [torch.zeros((visible_cap, 2), dtype=f32, device=device),
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
          torch.zeros((max(temp_bytes, 1),), dtype=torch.uint8, device=device)]
    ws += [torch.zeros((1,), dtype=i32 if k in (16, 20) else (i64 if k in (17, 18, 19) else f32), device=device)
           for k in range(15, 22)]
    ws += [torch.zeros((1, 6), dtype=f32, device=device), torch.zeros((1, 4), dtype=f32, device=device)]
    out = [torch.zeros((batch, h, w, 3), dtype=f32, device=device),
           torch.zeros((batch, h, w, 1), dtype=f32, device=device),
           torch.zeros((batch, h, w, 1), dtype=f32, device=device),
           torch.zeros((batch, h, w, 1), dtype=i64, device=device)]
    cams = [rig.viewmats.to(device).contiguous(), rig.intrinsics.to(device).contiguous(),
            torch.eye(4, device=device).repeat(batch, 1, 1).contiguous(),
            torch.zeros((batch,), dtype=i64, device=device), torch.empty((0,), dtype=i64, device=device)]
    scene_tensors = [means, covariances, opacities, features, semantic,
                     torch.zeros((1,), dtype=i64, device=device), torch.tensor([0, g], dtype=i64, device=device)]

    def render():
        return ref.render(scene_tensors, cams, out, ws, h, w, g, 0.01, 100.0, 3.33, 0.3, False, 0.01, False,
                          ts, 4096, 64, False, False, False, False, deterministic, True, False)

    for _ in range(3):
        render()
    torch.cuda.synchronize()
    counters = ws[13].cpu().tolist()
    if counters[2] or counters[3]:
        raise RuntimeError(f"reference workspace overflowed: {counters}")
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record()
    for _ in range(frames):
        render()
    stop.record()
    torch.cuda.synchronize()
    return start.elapsed_time(stop) / frames, counters, [t.clone() for t in out]


def b200_frame(scene, rig, device, frames: int):
    backend = CustomCudaBackend(output_srgb=False, tile_size=16, deterministic=True)
    service = RendererService(backend, height=rig.height, width=rig.width, max_views=rig.viewmats.shape[0])
    service.initialize(stage=None, device=device)
    service.load_scene(0, **scene.to(device).as_kwargs())
    vm, k = rig.viewmats.to(device), rig.intrinsics.to(device)
    ids = torch.zeros((vm.shape[0],), dtype=torch.int64, device=device)
    for _ in range(3):
        out = service.render(vm, k, ids)
    torch.cuda.synchronize()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record()
    for _ in range(frames):
        out = service.render(vm, k, ids)
    stop.record()
    torch.cuda.synchronize()
    return start.elapsed_time(stop) / frames, backend.read_counters(), {n: t.clone() for n, t in out.items()}


def main() -> None:
    parser = argparse.ArgumentParser()
    parser.add_argument("--frames", type=int, default=10)
    parser.add_argument("--out", type=Path, default=None)
    args = parser.parse_args()
    device = torch.device("cuda")
    ref = load_reference_module("vgr_reference_camera")
    scene, rig = batched_workload()
    pixels = rig.viewmats.shape[0] * rig.height * rig.width
    ours_ms, ours_counters, ours_out = b200_frame(scene, rig, device, args.frames)
    result = {"workload": "batched-1m-rgb (1M Gaussians, features[0..2] as linear RGB, 64 cameras 640x480, tile 16)",
              "b200": {"ms": round(ours_ms, 3), "mpix_per_s": round(pixels / ours_ms / 1e3, 1),
                       "visible": ours_counters["visible_gaussians"],
                       "intersections": ours_counters["tile_intersections"]}}
    for deterministic in (True, False):
        ms, counters, out = reference_frame(ref, scene, rig, device, deterministic, args.frames)
        rgb_err = (out[0] - ours_out["rgb"]).abs().amax(dim=-1)
        result["reference_deterministic" if deterministic else "reference_global_radix"] = {
            "ms": round(ms, 3), "mpix_per_s": round(pixels / ms / 1e3, 1), "visible": counters[0],
            "intersections": counters[1], "rgb_max_abs_vs_b200": float(rgb_err.max()),
            "pixels_rgb_over_1e-4": int((rgb_err > 1e-4).sum()), "pixels": pixels,
            "rgb_mean_abs_vs_b200": float((out[0] - ours_out["rgb"]).abs().mean()),
            "alpha_max_abs_vs_b200": float((out[2] - ours_out["alpha"]).abs().max()),
            "semantic_agreement": float((out[3] == ours_out["semantic_id"]).float().mean()),
        }
        del out
        torch.cuda.empty_cache()
    line = json.dumps(result)
    print(line)
    if args.out:
        args.out.parent.mkdir(parents=True, exist_ok=True)
        args.out.write_text(line + "\n")


if __name__ == "__main__":
    main()
