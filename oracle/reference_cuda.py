"""The reference's own CUDA path, timed on this machine's GPU.

TEST INFRASTRUCTURE ONLY (imported by bench.py's reference arm).  It runs the
reference unchanged: its Python service and backend classes (the pure-Python
package installed under baseline/_ref by ``python -m pip install --no-deps
--target baseline/_ref <reference checkout>``) driving its CUDA extensions
compiled from its sources by oracle/build_ref.py (oracle/_ref/
vgr_reference_camera.so, vgr_reference_lidar.so), injected through the
backends' ``native_module=`` seam (cuda_backend.py:123-124,
cuda_lidar_backend.py:79-80).  The reference renders features[0..2] as
linear RGB (renderer_cuda.cu:2160-2164), so its camera figures are for the
degree-0 equation; bench.py's own arm reports this library on the same
equation beside them.

Each timing calibrates first (the reference's adaptive capacity grows its
workspace and validates), then switches to explicit capacity mode and times
frames with CUDA events, then checks the counters for overflow.
"""

from __future__ import annotations

import sys
import types
from pathlib import Path

import torch

ROOT = Path(__file__).resolve().parents[1]
BASELINE = ROOT / "baseline" / "_ref"
REF_SO = ROOT / "oracle" / "_ref"


def unavailable_reason() -> str | None:
    """None when the reference package and both built extensions are here."""
    if not torch.cuda.is_available():
        return "no CUDA device"
    for name in ("vgr_reference_camera", "vgr_reference_lidar"):
        if not (REF_SO / f"{name}.so").exists():
            return f"oracle/_ref/{name}.so not built (oracle/build_ref.py)"
    try:
        package()
    except ImportError as error:
        return f"reference Python package not installed under baseline/_ref ({error})"
    return None


def package():
    """The reference's Python package (plyfile, used only by its PLY loader,
    is stubbed when absent)."""
    if BASELINE.is_dir() and str(BASELINE) not in sys.path:
        sys.path.append(str(BASELINE))
    if "plyfile" not in sys.modules:
        try:
            import plyfile  # noqa: F401
        except ImportError:
            stub = types.ModuleType("plyfile")
            stub.PlyData = stub.PlyElement = object
            sys.modules["plyfile"] = stub
    import isaacsim_gaussian_renderer as ref

    return ref


def _modules():
    from oracle.build_ref import load_reference_module

    return load_reference_module("vgr_reference_camera"), load_reference_module("vgr_reference_lidar")


def _rgb_scene(scene, device):
    """A scene's tensors with features cut to the three linear-RGB channels
    the reference reads."""
    kw = scene.to(device).as_kwargs()
    kw["features"] = kw["features"][:, :3].contiguous()
    return kw


def _time(fn, frames: int, device) -> float:
    stream = torch.cuda.current_stream(device)
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(stream)
    for k in range(frames):
        fn(k)
    stop.record(stream)
    torch.cuda.synchronize(device)
    return start.elapsed_time(stop) / frames


def camera_groups(scenes, groups, intrinsics, scene_ids, poses, device, frames: int, warmup: int = 2):
    """Render every frame of ``poses`` [F, B, 4, 4] as one reference
    ``RendererService.render`` call per resolution group (the reference
    renders one resolution per service), all ``scenes`` registered in each.
    ``groups`` maps (height, width) -> camera indices.  Returns ms per
    frame and the summed device counters of the last frame."""
    ref = package()
    camera_module, _ = _modules()
    from isaacsim_gaussian_renderer.cuda_backend import CustomCudaBackend

    services = []
    for (h, w), cams in groups.items():
        idx = torch.tensor(cams, device=device)
        backend = CustomCudaBackend(native_module=camera_module, output_srgb=False, tile_size=16)
        service = ref.RendererService(backend, height=h, width=w, max_views=len(cams))
        service.initialize(stage=None, device=device)
        for sid, scene in scenes:
            service.load_scene(sid, **_rgb_scene(scene, device))
        group = (service, backend, poses[:, idx].contiguous(), intrinsics[idx].contiguous(),
                 scene_ids[idx].contiguous(), service.prepare_outputs(len(cams)))
        service.render(group[2][0], group[3], group[4], outputs=group[5])  # calibration (grows)
        backend.adaptive_capacity = False
        services.append(group)

    def frame(k: int) -> None:
        for service, _, gp, gi, gs, out in services:
            service.render(gp[k % gp.shape[0]], gi, gs, outputs=out)

    for k in range(warmup):
        frame(k)
    torch.cuda.synchronize(device)
    ms = _time(frame, frames, device)
    totals = {"visible_gaussians": 0, "tile_intersections": 0, "overflow": 0}
    for _, backend, *_ in services:
        counters = backend.read_counters()
        totals["visible_gaussians"] += counters["visible_gaussians"]
        totals["tile_intersections"] += counters["tile_intersections"]
        totals["overflow"] += counters["visible_overflow"] + counters["intersection_overflow"]
    outputs = [group[5] for group in services]
    for service, *_ in services:
        service.shutdown()
    return ms, totals, outputs


def lidar_frames(work, device, frames: int, moved_means, far_plane_m: float, packet: int):
    """The reference's GaussianLidarService on its own CUDA build: every frame
    writes moved means into the scene's storage, revises the scene (the
    reference's LBVH rebuild) and traces every ray.  Returns (ms per frame,
    returns found in the last frame)."""
    ref = package()
    _, lidar_module = _modules()
    from isaacsim_gaussian_renderer.cuda_lidar_backend import CudaLidarBackend

    sensors = work.sensor_to_world.shape[0]
    rays = work.ray_directions.shape[0]
    backend = CudaLidarBackend(native_module=lidar_module, far_plane_m=far_plane_m, packet_size=packet)
    service = ref.GaussianLidarService(backend, max_sensors=sensors, max_rays=rays, returns=1)
    service.initialize(stage=None, device=device)
    scene = work.scene_kwargs(device)
    means = scene["means"]
    service.load_scene(0, **scene)
    dirs = work.ray_directions.to(device)
    times = work.time_offsets_ns.to(device)
    poses = work.sensor_to_world.to(device)
    ids = torch.zeros((sensors,), dtype=torch.int64, device=device)
    outputs = service.render_lidar(dirs, times, poses, ids)
    revision = [0]

    def frame(k: int) -> None:
        means.copy_(moved_means[k % len(moved_means)], non_blocking=True)
        revision[0] += 1
        service.revise_scene(0, revision=revision[0])
        service.render_lidar(dirs, times, poses, ids, outputs=outputs)

    for k in range(2):
        frame(k)
    torch.cuda.synchronize(device)
    ms = _time(frame, frames, device)
    found = int(outputs["valid"].sum().item())
    service.shutdown()
    return ms, found
