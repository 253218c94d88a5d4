"""Golden record of where the reference's CUDA build and the oracle differ at
full size, for the threshold-flip check.

Runs on a CUDA machine with the reference's CUDA build
(oracle/_ref/vgr_reference_camera.so, oracle/build_ref.py) and its Python
package (baseline/_ref).  Case: the batched workload's 1M-Gaussian scene
with features[0..2] as linear RGB (the reference's equation), cameras 0, 16,
32 and 48 of its 64-camera orbit at 640x480, tile 16, deterministic order,
rendered by the reference's RendererService + CustomCudaBackend on its own
CUDA build, and by the CPU oracle (with per-pixel decision margins).
Stored in tests/golden/camera_threshold_flips.npz: every pixel whose RGB
differs by more than 1e-4 (flat index, both values, the oracle's margins),
the largest difference elsewhere, and both frames' counters.  The inputs
are regenerated from the seeds by the test.

Usage: python tests/golden/make_threshold_golden.py [--out DIR]
"""

from __future__ import annotations

import argparse
import os
import sys
from pathlib import Path

import numpy as np
import torch

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT / "vectorized-gaussian-renderer-public_b200"))
sys.path.insert(0, str(ROOT))

from oracle import camera as oc  # noqa: E402
from oracle import reference_cuda  # noqa: E402
from vgr_b200.workloads import CameraRig, batched_workload  # noqa: E402

CAMERAS = (0, 16, 32, 48)


def case():
    scene, rig = batched_workload()
    idx = list(CAMERAS)
    rig = CameraRig(rig.viewmats[idx].contiguous(), rig.intrinsics[idx].contiguous(), rig.height, rig.width)
    return scene, rig


def oracle_frame(scene, rig, with_margins=True):
    feats = scene.features[:, :3].contiguous().numpy()
    return oc.render(
        means=scene.means.numpy(),
        covariances=oc.precompute_covariances(scene.scales.numpy(), scene.rotations.numpy()),
        opacities=scene.opacities.numpy(), features=feats, semantic_ids=scene.semantic_ids.numpy(),
        registered_scene_ids=[0], scene_offsets=[0, scene.means.shape[0]],
        viewmats=rig.viewmats.numpy(), intrinsics=rig.intrinsics.numpy(),
        camera_scene_ids=[0] * rig.viewmats.shape[0], height=rig.height, width=rig.width,
        sh_degree=-1, threads=os.cpu_count() or 1, with_margins=with_margins,
    )


def main() -> None:
    parser = argparse.ArgumentParser()
    parser.add_argument("--out", type=Path, default=ROOT / "tests" / "golden")
    args = parser.parse_args()
    reason = reference_cuda.unavailable_reason()
    if reason:
        raise SystemExit(f"reference CUDA path unavailable: {reason}")
    ref = reference_cuda.package()
    camera_module, _ = reference_cuda._modules()
    from isaacsim_gaussian_renderer.cuda_backend import CustomCudaBackend

    scene, rig = case()
    device = torch.device("cuda")
    backend = CustomCudaBackend(native_module=camera_module, output_srgb=False, deterministic=True)
    service = ref.RendererService(backend, height=rig.height, width=rig.width, max_views=len(CAMERAS))
    service.initialize(stage=None, device=device)
    kw = scene.to(device).as_kwargs()
    kw["features"] = kw["features"][:, :3].contiguous()
    service.load_scene(0, **kw)
    out = service.render(rig.viewmats.to(device), rig.intrinsics.to(device),
                         torch.zeros((len(CAMERAS),), dtype=torch.int64, device=device))
    service.synchronize()
    counters = backend.read_counters()
    ref_rgb = out["rgb"].cpu().numpy().reshape(-1, 3)
    ref_sem = out["semantic_id"].cpu().numpy().reshape(-1)
    got = oracle_frame(scene, rig)
    rgb = got.rgb.reshape(-1, 3)
    diff = np.abs(rgb - ref_rgb).max(axis=1)
    flagged = np.nonzero(diff > 1e-4)[0]
    margins = got.margins.reshape(-1, 3)
    np.savez_compressed(
        args.out / "camera_threshold_flips.npz",
        cameras=np.array(CAMERAS),
        flagged=flagged.astype(np.int64),
        reference_rgb=ref_rgb[flagged],
        oracle_rgb=rgb[flagged],
        oracle_margins=margins[flagged],
        max_abs_elsewhere=np.float32(np.delete(diff, flagged).max() if flagged.size < diff.size else 0.0),
        pixels=np.int64(diff.size),
        semantic_disagreements=np.int64((ref_sem != got.semantic.reshape(-1)).sum()),
        reference_counters=np.array([counters["visible_gaussians"], counters["tile_intersections"]]),
        oracle_counters=np.array([got.visible, got.intersections]),
    )
    small = (margins.min(axis=1) < 1e-4).mean()
    print(f"flagged {flagged.size} of {diff.size}; max elsewhere {np.delete(diff, flagged).max():.3g}; "
          f"pixels with a margin below 1e-4: {small:.4f}; counters ref {counters['visible_gaussians']}, "
          f"{counters['tile_intersections']} oracle {got.visible}, {got.intersections}")
    for k in flagged[:40]:
        print(k, diff[k], margins[k])
    service.shutdown()


if __name__ == "__main__":
    main()
