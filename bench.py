#!/usr/bin/env python
"""Benchmark of the B200 batched Gaussian-splat sensor renderer.

python bench.py [--gpus N --steps K --warmup W] [--impl b200|reference]

Headline workload (ragged-8scenes-1024cams): eight scenes of 100k..3M
Gaussians (9.1M in all, degree-3 spherical harmonics), 1,024 cameras split
32..256 per scene at mixed resolutions 128x128 / 160x120 / 320x240, a pose
sequence with small per-frame deltas; seeded synthetic data of those laws (no
dataset).  One step is one ragged frame: every camera, all four outputs, as
one submission replayed from a CUDA graph.  ``value`` is Mpix/s with the
inputs resident in HBM (scenes of 2.2 GB, far above L2); ``e2e`` is the same
frame through the C-ABI ragged entry point with the poses copied from pinned
host memory and every output copied back to pinned host memory inside the
timed region.  Beside it, top-level keys give the plain form on the same
frames (one render per resolution, the reference's drop-in form) and the
ratio, the batched 1M-Gaussian 64-camera frame, the differentiable training
step and the LiDAR frame.  ``roofline`` is for the ragged frame's kernel with
the largest device time, timed live with CUDA events between its stages;
``cpu_baseline`` times the CPU oracle on a bounded camera sample.

Under torchrun (N > 1) the ragged frame is split across ranks by estimated
work (pixels and tile intersections per camera, from one calibration frame
that every rank renders): each rank renders a contiguous run of cameras
against its own replica of the scenes, with no collective on the data path;
the frame time is the max over ranks, so the scaling is strong.

``--impl reference`` times the reference's CPU path (the CPU oracle: the
reference has no CPU renderer, so this is the restatement of its equation)
on a camera sample of the same ragged frames, and beside it, when the
reference's package and CUDA build are present, the reference's own CUDA
path on the same box: the ragged frames, the batched frame and the LiDAR
frame.
"""

from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "vectorized-gaussian-renderer-public_b200"))
sys.path.insert(0, str(ROOT))

import numpy as np  # noqa: E402
import torch  # noqa: E402

METRIC = "Mpix/s ragged batch + fwd+bwd ms/iter, chosen vs plain form at 1e-4 RGB err"
UNIT = "Mpix/s"
STAGES = ("setup", "project_emit", "tile_scan", "bucket_scatter", "tile_sort", "composite")
KERNEL_NAMES = {
    "setup": "camera_setup_kernel",
    "project_emit": "project_emit_kernel",
    "tile_scan": "tile_scan_kernel",
    "bucket_scatter": "bucket_scatter_kernel",
    "tile_sort": "tile_sort_kernel",
    "composite": "composite_kernel",
}
FALLBACK_HBM_GBS = 6650.0
RAGGED_WORKLOAD = "ragged-8scenes-1024cams"


def parse_args() -> argparse.Namespace:
    parser = argparse.ArgumentParser()
    parser.add_argument("--gpus", type=int, default=1)
    parser.add_argument("--steps", type=int, default=20, help="timed ragged frames")
    parser.add_argument("--warmup", type=int, default=5)
    parser.add_argument("--impl", choices=("b200", "reference"), default="b200")
    parser.add_argument("--cpu-sample-cameras", type=int, default=16,
                        help="ragged cameras the CPU oracle renders per step (two per scene)")
    parser.add_argument("--no-cpu-baseline", action="store_true")
    parser.add_argument("--no-e2e", action="store_true")
    parser.add_argument("--ragged-scale", type=float, default=1.0,
                        help="scale scene sizes and camera counts of the ragged workload (small captures)")
    parser.add_argument("--plain-steps", type=int, default=5, help="plain-form frames (0: skip)")
    parser.add_argument("--rgb-steps", type=int, default=10,
                        help="frames of the ragged workload on the linear-RGB equation (0: skip)")
    parser.add_argument("--tile", type=int, default=None,
                        help="fix the ragged tile size instead of autotuning (profiling captures)")
    parser.add_argument("--composite-shape", type=int, default=None, choices=(0, 1, 2),
                        help="compositor CTA shape with --tile, and for the batched workload")
    parser.add_argument("--batched-steps", type=int, default=10,
                        help="frames of the batched 1M-Gaussian 64-camera workload (0: skip)")
    parser.add_argument("--cameras", type=int, default=None,
                        help="camera count of the batched workload (small profiling captures)")
    parser.add_argument("--lidar-steps", type=int, default=5,
                        help="LiDAR frames (0: skip)")
    parser.add_argument("--lidar-sensors", type=int, default=None,
                        help="override the LiDAR sensor count (small profiling captures)")
    parser.add_argument("--aux-steps", type=int, default=10,
                        help="timed steps of PLY ingestion and the hybrid compositor (0: skip)")
    parser.add_argument("--mode-steps", type=int, default=5,
                        help="frames per dense-mode / exact-ray measurement (0 skips)")
    parser.add_argument("--mode-cameras", type=int, default=None,
                        help="cameras of both mode workloads (default 32 deep-scene, 64 batched; small for ncu)")
    parser.add_argument("--diff-steps", type=int, default=10,
                        help="timed steps of the differentiable-form workload (0: skip)")
    parser.add_argument("--no-reference-cuda", action="store_true",
                        help="reference arm: skip the reference's CUDA timings")
    parser.add_argument("--detail", type=Path, default=None,
                        help="also write every section's full record to this JSON file")
    return parser.parse_args()


def measured_peaks() -> tuple[float, str]:
    path = ROOT / "MEASURED_PEAKS.json"
    try:
        data = json.loads(path.read_text())
        return float(data["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def recorded_traffic(workload: str) -> dict:
    """Per-launch DRAM bytes from committed ncu summaries, if present."""
    path = ROOT / "profiles" / "traffic.json"
    try:
        return json.loads(path.read_text()).get(workload, {})
    except Exception:
        return {}


# --------------------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons while timing."""

    FIELDS = (
        "clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
        "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
        "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"
    )

    def __init__(self, index: int) -> None:
        self.index = index
        self.proc: subprocess.Popen | None = None
        self.lines: list[str] = []
        self.thread: threading.Thread | None = None

    def start(self) -> None:
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True,
            )
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._pump, daemon=True)
        self.thread.start()

    def _pump(self) -> None:
        assert self.proc is not None and self.proc.stdout is not None
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread is not None:
            self.thread.join(timeout=5)
        sm, sm_max, power, reasons = [], [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                sm_max.append(float(parts[1]))
                power.append(float(parts[2]))
            except ValueError:
                continue
            for name, flag in zip(names, parts[4:8]):
                if flag.lower() == "active":
                    reasons.add(name)
        under_load = sorted(sm)[len(sm) // 2:] if sm else []
        return {
            "sm_mhz": statistics.median(under_load) if under_load else None,
            "sm_max_mhz": max(sm_max) if sm_max else None,
            "power_w_max": max(power) if power else None,
            "samples": len(sm),
            "reasons": sorted(reasons),
        }


# --------------------------------------------------------------------------- distributed
def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def max_over_ranks(value: float, world: int, device) -> float:
    if world == 1:
        return value
    import torch.distributed as dist

    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world: int) -> None:
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


# --------------------------------------------------------------------------- workload description
def ragged_config(work, frames: int) -> dict:
    """The ragged workload's description, identical in both arms."""
    groups: dict[str, int] = {}
    for h, w in zip(work.heights, work.widths):
        groups[f"{w}x{h}"] = groups.get(f"{w}x{h}", 0) + 1
    return {
        "workload": RAGGED_WORKLOAD,
        "scene_gaussians": [s.means.shape[0] for _, s in work.scenes],
        "cameras": len(work.heights),
        "cameras_per_resolution": groups,
        "pixels_per_frame": sum(h * w for h, w in zip(work.heights, work.widths)),
        "sh_degree": 3,
        "outputs": "rgb, depth, alpha, semantic_id",
        "frames": frames,
        "l2": "inputs larger than L2 (scenes 2.2 GB)",
    }


def ragged_frames(args) -> int:
    """Pose frames generated: the workload's 100-frame sequence, or more
    when warm-up and timed frames need them."""
    return max(100, max(args.warmup, 0) + max(args.steps, 1))


def group_by_resolution(work, cams=None) -> dict[tuple[int, int], list[int]]:
    groups: dict[tuple[int, int], list[int]] = {}
    for c in (range(len(work.heights)) if cams is None else cams):
        groups.setdefault((work.heights[c], work.widths[c]), []).append(c)
    return groups


def cpu_sample_cameras(work, count: int) -> list[int]:
    """``count`` cameras spread over the scenes: the first cameras of each
    scene in turn (cameras are grouped by scene)."""
    ids = work.scene_ids.tolist()
    firsts = {}
    for c, sid in enumerate(ids):
        firsts.setdefault(sid, []).append(c)
    picked: list[int] = []
    k = 0
    while len(picked) < count and any(k < len(v) for v in firsts.values()):
        for sid in sorted(firsts):
            if k < len(firsts[sid]) and len(picked) < count:
                picked.append(firsts[sid][k])
        k += 1
    return sorted(picked)


# --------------------------------------------------------------------------- CPU path
class RaggedOracle:
    """The CPU oracle over the ragged scenes (all registered, covariances
    precomputed once), rendering camera subsets of the ragged frames."""

    def __init__(self, work) -> None:
        from oracle import camera as oc

        self.oc = oc
        self.work = work
        scenes = [s for _, s in work.scenes]
        self.kwargs = dict(
            means=np.concatenate([s.means.numpy() for s in scenes]),
            covariances=oc.precompute_covariances(np.concatenate([s.scales.numpy() for s in scenes]),
                                                  np.concatenate([s.rotations.numpy() for s in scenes])),
            opacities=np.concatenate([s.opacities.numpy() for s in scenes]),
            features=np.concatenate([s.features.numpy() for s in scenes]),
            semantic_ids=np.concatenate([s.semantic_ids.numpy() for s in scenes]),
            registered_scene_ids=np.array([sid for sid, _ in work.scenes], dtype=np.int64),
            scene_offsets=np.cumsum([0] + [s.means.shape[0] for s in scenes]).astype(np.int64),
        )

    def render(self, cams: list[int], frame: int, threads: int):
        w = self.work
        heights = [w.heights[c] for c in cams]
        widths = [w.widths[c] for c in cams]
        ragged = dict(
            widths=widths, heights=heights,
            tile_offsets=np.cumsum([0] + [-(-h // 16) * -(-x // 16) for h, x in zip(heights, widths)]),
            pixel_offsets=np.cumsum([0] + [h * x for h, x in zip(heights, widths)]),
        )
        result = self.oc.render(
            **self.kwargs, viewmats=w.viewmats[frame % w.viewmats.shape[0]].numpy()[cams],
            intrinsics=w.intrinsics.numpy()[cams], camera_scene_ids=w.scene_ids.numpy()[cams],
            height=max(heights), width=max(widths), sh_degree=3, threads=threads, ragged=ragged,
        )
        return result, int(ragged["pixel_offsets"][-1])


def time_ragged_cpu(work, cams: list[int], steps: int, warmup: int) -> tuple[float, float, int, str]:
    """Mpix/s of the CPU oracle rendering ``cams`` of the ragged frames,
    one frame per step, on every host core."""
    threads = os.cpu_count() or 1
    oracle = RaggedOracle(work)
    for k in range(min(warmup, 1)):
        oracle.render(cams[:1], k, threads)
    pixels = 0
    start = time.perf_counter()
    for k in range(steps):
        _, px = oracle.render(cams, k, threads)
        pixels += px
    seconds = time.perf_counter() - start
    sample = (f"{len(cams)} of {len(work.heights)} cameras per frame (two per scene, all three resolutions, "
              f"{pixels // max(steps, 1)} px), full scenes, {steps} frames")
    return pixels / seconds / 1e6, seconds, threads, sample


# --------------------------------------------------------------------------- algorithmic bytes
def camera_stage_bytes(g_total: int, feature_floats: int, visible: int, isects: int, tiles: int,
                       pixels: int, cameras: int) -> dict[str, float]:
    """Algorithmic bytes per launch of each camera stage, counted per unit of
    work: the scene read once per frame
    (G x (12 mean + 16 quaternion + 12 scale + 4 opacity + 8 semantic + 4F)),
    a 48-byte record written once by the projection and read once by the
    compositor, 12 bytes of key + value per intersection at emission, the
    sort's own passes over the intersections (scatter: key + value read,
    8-byte bucket entry written; tile sort: entry read, key + value
    written), the compositor's 4-byte value per intersection and 28 bytes of
    outputs per pixel."""
    scene = g_total * (12 + 16 + 12 + 4 + 8 + 4 * feature_floats)
    return {
        "setup": cameras * (64 + 36 + 64 + 8 + 176),
        "project_emit": scene + visible * 48 + isects * 12,
        "tile_scan": tiles * (4 + 8),
        "bucket_scatter": isects * (12 + 8),
        "tile_sort": isects * (8 + 12),
        "composite": isects * 4 + visible * 48 + pixels * 28,
    }


def roofline_of(stage_avg: dict[str, float], stage_bytes: dict[str, float], workload: str) -> dict:
    dominant = max(stage_avg, key=stage_avg.get)
    peak, peak_kind = measured_peaks()
    traffic = recorded_traffic(workload)
    achieved = stage_bytes[dominant] / (stage_avg[dominant] / 1e3) / 1e9
    kernel = KERNEL_NAMES[dominant]
    return {
        "bound": "hbm",
        "kernel": kernel,
        "achieved": round(achieved, 1),
        "peak": peak,
        "unit": "GB/s",
        "frac": round(achieved / peak, 4),
        "peak_source": f"hbm_gbs of {peak_kind}",
        "traffic": traffic.get(kernel),
        "traffic_source": traffic.get("_source"),
        "algorithmic_bytes": int(stage_bytes[dominant]),
        "ms": round(stage_avg[dominant], 4),
        "issue_active_ncu": traffic.get("_issue_active", {}).get(kernel),
    }


# --------------------------------------------------------------------------- ragged headline
def ragged_backend(work, device, sh_degree):
    from vgr_b200 import CustomCudaBackend, RendererService

    backend = CustomCudaBackend(sh_degree=sh_degree, output_srgb=False)
    holder = RendererService(backend, height=16, width=16, max_views=1)
    holder.initialize(stage=None, device=device)
    for sid, scene in work.scenes:
        kw = scene.to(device).as_kwargs()
        if sh_degree is None:
            kw["features"] = kw["features"][:, :3].contiguous()
        holder.load_scene(sid, **kw)
    return backend, holder


def run_ragged(args, device, world: int, rank: int, work) -> dict:
    """The headline: the ragged frame as one CUDA-graph submission per frame
    (the rank's share of the cameras under torchrun)."""
    from vgr_b200 import _native
    from vgr_b200.distributed import camera_costs, weighted_camera_shards
    from vgr_b200.ragged import RaggedBatch, autotune_tile_size

    lib = _native.load_library()
    frames = ragged_frames(args)
    stream = torch.cuda.current_stream(device)
    scene_ids = work.scene_ids.to(device)
    intr = work.intrinsics.to(device)
    poses = work.viewmats.to(device)
    backend, holder = ragged_backend(work, device, 3)

    cams = list(range(len(work.heights)))
    split = None
    if world > 1:
        # Every rank renders the whole first frame once, derives the same
        # per-camera costs and cuts the same contiguous shards.
        full = RaggedBatch(backend, work.heights, work.widths)
        out_full = full.outputs()
        full.calibrate(poses[0].contiguous(), intr, scene_ids, out_full)
        ws = full.workspace
        tile_offsets = [0]
        for h, w in zip(work.heights, work.widths):
            tile_offsets.append(tile_offsets[-1] + math.ceil(h / full.tile_size) * math.ceil(w / full.tile_size))
        costs = camera_costs(ws["tile_starts"], ws["tile_ends"], tile_offsets,
                             [h * w for h, w in zip(work.heights, work.widths)])
        shards = weighted_camera_shards(costs, world)
        cams = list(range(len(work.heights)))[shards[rank]]
        split = {"shard_cameras": [s.stop - s.start for s in shards],
                 "shard_cost_share": [round(sum(costs[s]) / max(sum(costs), 1e-9), 4) for s in shards]}
        del full, out_full, ws
        torch.cuda.empty_cache()
    idx = torch.tensor(cams, device=device)
    heights = [work.heights[c] for c in cams]
    widths = [work.widths[c] for c in cams]
    r_ids = scene_ids[idx].contiguous()
    r_intr = intr[idx].contiguous()
    r_poses = poses[:, idx].contiguous()
    pixels = sum(h * w for h, w in zip(heights, widths))

    ragged = RaggedBatch(backend, heights, widths)
    outputs = ragged.outputs()
    view = r_poses[0].clone()
    if args.tile:
        if args.composite_shape is not None:
            ragged.composite_shape = args.composite_shape
        ragged._set_tiles(args.tile)
        tile = args.tile
    else:
        tile = autotune_tile_size(ragged, view, r_intr, r_ids, outputs, candidates=(8, 16, 32),
                                  persistent_candidates=(False, True), shape_candidates=(0, 1, 2))
    counters = ragged.calibrate(view, r_intr, r_ids, outputs)
    launches0 = lib.vgr_kernel_launch_count()
    ragged.render(view, r_intr, r_ids, outputs)
    launches_per_frame = lib.vgr_kernel_launch_count() - launches0
    graph = ragged.capture(view, r_intr, r_ids, outputs)
    for k in range(max(args.warmup, 3)):
        view.copy_(r_poses[k % frames])
        graph.replay()
    torch.cuda.synchronize(device)

    sampler = ClockSampler(device.index if device.index is not None else 0)
    barrier(world)
    torch.cuda.synchronize(device)
    sampler.start()
    time.sleep(0.3)
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(stream)
    for k in range(args.steps):
        view.copy_(r_poses[(args.warmup + k) % frames])
        graph.replay()
    stop.record(stream)
    torch.cuda.synchronize(device)
    barrier(world)
    clocks = sampler.stop()
    elapsed = max_over_ranks(start.elapsed_time(stop), world, device)
    ms = elapsed / args.steps
    check = ragged.check()
    total_pixels = sum(h * w for h, w in zip(work.heights, work.widths))
    value = total_pixels / (ms / 1e3) / 1e6

    # Live stage times (eager frames with CUDA events at the stage boundaries).
    stage_runs = []
    for k in range(3):
        marks = [torch.cuda.Event(enable_timing=True) for _ in range(_native.STAGE_EVENTS)]
        ragged.set_stage_events(marks)
        view.copy_(r_poses[k % frames])
        ragged.render(view, r_intr, r_ids, outputs)
        ragged.set_stage_events(None)
        stage_runs.append(marks)
    torch.cuda.synchronize(device)
    stage_avg = {name: statistics.fmean(m[i].elapsed_time(m[i + 1]) for m in stage_runs)
                 for i, name in enumerate(STAGES)}
    g_total = sum(s.means.shape[0] for _, s in work.scenes)
    sbytes = camera_stage_bytes(g_total, 48, counters["visible_gaussians"], counters["tile_intersections"],
                                ragged.total_tiles, pixels, len(cams))
    roofline = roofline_of(stage_avg, sbytes, RAGGED_WORKLOAD)
    roofline["stage_ms"] = {k: round(v, 3) for k, v in stage_avg.items()}
    roofline["stage_frac_of_hbm"] = {
        k: round(sbytes[k] / (stage_avg[k] / 1e3) / 1e9 / roofline["peak"], 4) for k in STAGES if stage_avg[k] > 0
    }

    e2e = None
    if not args.no_e2e:
        e2e = ragged_e2e(args, device, world, ragged, r_poses, r_intr, r_ids, outputs, total_pixels)
    last = {name: t.clone() for name, t in outputs.items()}
    result = {
        "value": value, "ms": ms, "clocks": clocks, "roofline": roofline, "e2e": e2e,
        "launches": launches_per_frame * args.steps, "tile": tile,
        "persistent": bool(ragged.persistent_compositor), "shape": int(ragged.composite_shape),
        "autotune_ms": {str(k): round(v, 3) for k, v in ragged.autotune_ms.items()},
        "counters": counters, "overflow": bool(check["visible_overflow"] or check["intersection_overflow"]),
        "split": split, "cams": cams, "last": last, "ragged": ragged, "backend": backend, "holder": holder,
        "poses": r_poses, "intr": r_intr, "ids": r_ids,
    }
    return result


def ragged_e2e(args, device, world, ragged, poses, intr, ids, outputs, total_pixels) -> dict:
    """End to end through the C-ABI ragged entry point: per frame, poses from
    pinned host memory, the render, and every output back to pinned host
    memory, pipelined over two output sets (frame k's download on a copy
    stream overlaps frame k+1's render)."""
    stream = torch.cuda.current_stream(device)
    host_poses = poses.cpu().pin_memory()
    view = poses[0].clone()
    sets = [outputs, {name: torch.empty_like(t) for name, t in outputs.items()}]
    host_sets = [{name: torch.empty(t.shape, dtype=t.dtype, pin_memory=True) for name, t in outputs.items()}
                 for _ in range(2)]
    h2d = view.numel() * 4
    d2h = sum(t.numel() * t.element_size() for t in host_sets[0].values())
    steps = max(2, min(args.steps, 10))
    copy_stream = torch.cuda.Stream(device)

    def run(count: int) -> float:
        done = [None, None]
        torch.cuda.synchronize(device)
        barrier(world)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for k in range(count):
            b = k % 2
            if done[b] is not None:
                stream.wait_event(done[b])
            view.copy_(host_poses[k % host_poses.shape[0]], non_blocking=True)
            ragged.render(view, intr, ids, sets[b])
            rendered = torch.cuda.Event()
            rendered.record(stream)
            copy_stream.wait_event(rendered)
            with torch.cuda.stream(copy_stream):
                for name, t in sets[b].items():
                    host_sets[b][name].copy_(t, non_blocking=True)
            done[b] = torch.cuda.Event()
            done[b].record(copy_stream)
        for ev in done:
            if ev is not None:
                stream.wait_event(ev)
        e1.record(stream)
        torch.cuda.synchronize(device)
        return max_over_ranks(e0.elapsed_time(e1), world, device)

    run(2)
    e_ms = run(steps)
    for b in range(2):
        for name in outputs:
            if not torch.equal(host_sets[b][name].to(device), sets[b][name]):
                raise RuntimeError(f"e2e: downloaded {name} differs from the device output")
    return {
        "value": round(total_pixels * steps / (e_ms / 1e3) / 1e6, 3),
        "unit": UNIT,
        "h2d_bytes_per_step": h2d,
        "d2h_bytes_per_step": d2h,
        "steps": steps,
        "pipelined": "two output sets; frame k's download overlaps frame k+1's render",
    }


def run_plain(args, device, work, head: dict) -> dict:
    """The plain form on the same frames: one RendererService per
    resolution, every scene registered, one render call per resolution per
    frame (the fewest calls the plain form allows).  Its images must equal
    the ragged form's."""
    from vgr_b200 import CustomCudaBackend, RendererService

    frames = ragged_frames(args)
    stream = torch.cuda.current_stream(device)
    poses, intr, ids = head["poses"], head["intr"], head["ids"]
    cams = head["cams"]
    groups: dict[tuple[int, int], list[int]] = {}
    for j, c in enumerate(cams):
        groups.setdefault((work.heights[c], work.widths[c]), []).append(j)
    plain = []
    for (h, w), members in groups.items():
        idx = torch.tensor(members, device=device)
        b = CustomCudaBackend(sh_degree=3, output_srgb=False, tile_size=min(head["tile"], 16),
                              composite_shape=head["shape"])
        svc = RendererService(b, height=h, width=w, max_views=len(members))
        svc.initialize(stage=None, device=device)
        for sid, scene in work.scenes:
            svc.load_scene(sid, **scene.to(device).as_kwargs())
        gp, gi, gs = poses[:, idx].contiguous(), intr[idx].contiguous(), ids[idx].contiguous()
        out = svc.prepare_outputs(len(members))
        svc.render(gp[0], gi, gs, outputs=out)
        b.adaptive_capacity = False
        plain.append((svc, b, gp, gi, gs, out, members))

    def frame(k: int) -> None:
        for svc, _, gp, gi, gs, out, _ in plain:
            svc.render(gp[k % frames], gi, gs, outputs=out)

    for k in range(3):
        frame(k)
    torch.cuda.synchronize(device)
    steps = max(args.plain_steps, 1)
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(stream)
    for k in range(steps):
        frame(args.warmup + k)
    stop.record(stream)
    torch.cuda.synchronize(device)
    ms = start.elapsed_time(stop) / steps
    # Same frame both ways: re-render the ragged form's last frame eagerly.
    ragged, outputs = head["ragged"], head["last"]
    last = (args.warmup + args.steps - 1) % frames
    view = poses[last].contiguous()
    ragged.render(view, intr, ids, outputs)
    frame(last)
    torch.cuda.synchronize(device)
    max_abs = 0.0
    for *_, out, members in plain:
        for j, cam in enumerate(members):
            diff = (ragged.view(outputs, "rgb", cam) - out["rgb"][j]).abs().max().item()
            max_abs = max(max_abs, diff)
    overflow = any(b.check_capacity()["intersection_overflow"] or b.check_capacity()["visible_overflow"]
                   for _, b, *_ in plain)
    for svc, *_ in plain:
        svc.shutdown()
    pixels = sum(work.heights[c] * work.widths[c] for c in cams)
    return {"value": round(pixels / (ms / 1e3) / 1e6, 3), "ms_per_frame": round(ms, 3),
            "calls_per_frame": len(plain), "rgb_max_abs_vs_ragged": max_abs, "overflow": overflow}


def run_ragged_rgb(args, device, work) -> dict:
    """The ragged frames with features[0..2] as linear RGB (the reference's
    equation), for the same-box comparison with the reference's CUDA path."""
    from vgr_b200.ragged import RaggedBatch, autotune_tile_size

    backend, holder = ragged_backend(work, device, None)
    ids = work.scene_ids.to(device)
    intr = work.intrinsics.to(device)
    poses = work.viewmats.to(device)
    ragged = RaggedBatch(backend, work.heights, work.widths)
    outputs = ragged.outputs()
    view = poses[0].clone()
    autotune_tile_size(ragged, view, intr, ids, outputs, candidates=(16, 32))
    ragged.calibrate(view, intr, ids, outputs)
    graph = ragged.capture(view, intr, ids, outputs)
    stream = torch.cuda.current_stream(device)
    for k in range(3):
        view.copy_(poses[k])
        graph.replay()
    torch.cuda.synchronize(device)
    steps = max(args.rgb_steps, 2)
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(stream)
    for k in range(steps):
        view.copy_(poses[k % poses.shape[0]])
        graph.replay()
    stop.record(stream)
    torch.cuda.synchronize(device)
    ms = start.elapsed_time(stop) / steps
    ragged.check()
    holder.shutdown()
    pixels = sum(h * w for h, w in zip(work.heights, work.widths))
    return {"value": round(pixels / (ms / 1e3) / 1e6, 1), "ms_per_frame": round(ms, 3), "tile": ragged.tile_size}


# --------------------------------------------------------------------------- batched 1M frame
def run_batched(args, device) -> dict:
    """Batched frame: 1M Gaussians SH3, 64 cameras 640x480, through
    RendererService (one call per frame); per-stage times and the
    compositor's roofline."""
    from vgr_b200 import CustomCudaBackend, RendererService, _native
    from vgr_b200.workloads import batched_workload

    count = args.cameras or 64
    scene, rig = batched_workload(cameras=count)

    def frame_ms(sh_degree, with_stages: bool):
        shape = {} if args.composite_shape is None else {"composite_shape": args.composite_shape}
        backend = CustomCudaBackend(sh_degree=sh_degree, output_srgb=False, tile_size=16, **shape)
        service = RendererService(backend, height=rig.height, width=rig.width, max_views=count)
        service.initialize(stage=None, device=device)
        kw = scene.to(device).as_kwargs()
        if sh_degree is None:
            kw["features"] = kw["features"][:, :3].contiguous()
        service.load_scene(0, **kw)
        view, intr = rig.viewmats.to(device), rig.intrinsics.to(device)
        ids = torch.zeros((count,), dtype=torch.int64, device=device)
        out = service.prepare_outputs(count)
        service.render(view, intr, ids, outputs=out)
        counters = backend.read_counters()
        backend.adaptive_capacity = False
        for _ in range(3):
            service.render(view, intr, ids, outputs=out)
        torch.cuda.synchronize(device)
        steps = max(args.batched_steps, 1)
        events = [[torch.cuda.Event(enable_timing=True) for _ in range(_native.STAGE_EVENTS)] for _ in range(steps)]
        stream = torch.cuda.current_stream(device)
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record(stream)
        for k in range(steps):
            if with_stages:
                backend.set_stage_events(events[k])
            service.render(view, intr, ids, outputs=out)
        stop.record(stream)
        torch.cuda.synchronize(device)
        backend.set_stage_events(None)
        ms = start.elapsed_time(stop) / steps
        overflow = backend.check_capacity()
        stages = None
        if with_stages:
            stages = {name: statistics.fmean(ev[i].elapsed_time(ev[i + 1]) for ev in events)
                      for i, name in enumerate(STAGES)}
        service.shutdown()
        return ms, counters, stages, bool(overflow["visible_overflow"] or overflow["intersection_overflow"])

    ms, counters, stages, overflow = frame_ms(3, True)
    pixels = count * rig.height * rig.width
    tiles = count * math.ceil(rig.height / 16) * math.ceil(rig.width / 16)
    sbytes = camera_stage_bytes(scene.means.shape[0], 48, counters["visible_gaussians"],
                                counters["tile_intersections"], tiles, pixels, count)
    peak, _ = measured_peaks()
    comp = sbytes["composite"] / (stages["composite"] / 1e3) / 1e9
    rgb_ms, _, _, _ = frame_ms(None, False)
    return {
        "workload": f"batched-1m-sh3 (1M Gaussians SH3, {count} cameras 640x480)",
        "value": round(pixels / (ms / 1e3) / 1e6, 1), "ms_per_frame": round(ms, 3),
        "stage_ms": {k: round(v, 3) for k, v in stages.items()},
        "composite_frac_of_hbm": round(comp / peak, 4),
        "visible_records": counters["visible_gaussians"], "tile_intersections": counters["tile_intersections"],
        "overflow": overflow,
        "rgb_equation": {"value": round(pixels / (rgb_ms / 1e3) / 1e6, 1), "ms_per_frame": round(rgb_ms, 3)},
    }


# --------------------------------------------------------------------------- LiDAR
LIDAR_METRIC = "rays/s, LBVH rebuilt every frame"
LIDAR_CONFIG = {"workload": "lidar-2m-64x128x2048", "gaussians": 2_000_000, "sensors": 64, "beams": 128,
                "azimuths": 2048, "returns": 1, "far_plane_m": 80.0, "packet": 8,
                "motion": "5% of means moved by N(0, 0.05) m before each frame's rebuild"}


def lidar_moved_means(means: torch.Tensor, seed: int) -> torch.Tensor:
    """``means`` with a seeded 5% subset moved by N(0, 0.05) m."""
    gen = torch.Generator().manual_seed(seed)
    count = means.shape[0]
    pick = torch.randperm(count, generator=gen)[: count // 20]
    moved = means.clone()
    moved[pick] += torch.randn((pick.numel(), 3), generator=gen) * 0.05
    return moved.contiguous()


def lidar_cpu_sample(work, rays_stride: int = 256, threads: int | None = None) -> tuple[float, int, str]:
    """Rays/s of the LiDAR CPU oracle on sensor 0 and every ``rays_stride``-th ray."""
    from oracle import lidar as ol

    threads = threads or os.cpu_count() or 1
    dirs = work.ray_directions.double().numpy()[::rays_stride]
    times = work.time_offsets_ns.numpy()[::rays_stride]
    scene = {
        "means": work.means.double().numpy(), "scales": work.scales.double().numpy(),
        "rotations": work.rotations.double().numpy(), "opacities": work.opacities.double().numpy(),
        "semantic_ids": work.semantic_ids.numpy(), "reflectivity": work.reflectivity.double().numpy(),
        "surface_confidence": None,
    }
    config = ol.LidarConfig(far_plane_m=LIDAR_CONFIG["far_plane_m"])
    sensors = work.sensor_to_world.double().numpy()[:1]
    start = time.perf_counter()
    ol.render({0: scene}, dirs, times, sensors, np.zeros(1, dtype=np.int64), returns=1, config=config,
              threads=threads)
    seconds = time.perf_counter() - start
    rays = dirs.shape[0]
    return rays / seconds, threads, f"sensor 0, {rays} of {work.ray_directions.shape[0]} rays, full 2M scene"


# --------------------------------------------------------------------------- ingestion / hybrid
def run_aux(args, device, world: int) -> dict:
    """Scene ingestion and the hybrid compositor, the two HBM-bound passes
    beside the hot path: PLY canonicalisation of a 1M-Gaussian SH3 vertex
    block already on the device (248 B read + 240 B written per Gaussian),
    and the Gaussian/mesh composite of two 64 x 640x480 layers (40 B read +
    21 B written per pixel)."""
    import numpy as np

    from vgr_b200 import _native
    from vgr_b200.hybrid_compositor import composite_gaussian_and_mesh
    from vgr_b200.ply import PlyVertexBlock, _layout

    peak, peak_source = measured_peaks()
    steps = max(args.aux_steps, 1)
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    stream = torch.cuda.current_stream(device)
    # PLY rows: x y z nx ny nz f_dc_0..2 f_rest_0..44 opacity scale_0..2 rot_0..3, float32.
    count = 1_000_000
    names = ["x", "y", "z", "nx", "ny", "nz", "f_dc_0", "f_dc_1", "f_dc_2"] + [f"f_rest_{i}" for i in range(45)]
    names += ["opacity", "scale_0", "scale_1", "scale_2", "rot_0", "rot_1", "rot_2", "rot_3"]
    gen = torch.Generator().manual_seed(17)
    rows = torch.randn((count, len(names)), generator=gen).to(device)
    block = PlyVertexBlock(count=count, properties=[(n, "float") for n in names],
                           body=np.zeros(0, np.uint8), row_bytes=4 * len(names))
    layout, width = _layout(block)
    outs = [torch.empty((count, 3), device=device), torch.empty((count, 3), device=device),
            torch.empty((count, 4), device=device), torch.empty((count,), device=device),
            torch.empty((count, width), device=device), torch.empty((count,), dtype=torch.int64, device=device)]
    lib = _native.load_library()

    def ingest() -> None:
        _native.check(lib.vgr_ply_canonicalize(rows.data_ptr(), count, layout, outs[0].data_ptr(), outs[1].data_ptr(),
                                               outs[2].data_ptr(), outs[3].data_ptr(), outs[4].data_ptr(), width,
                                               outs[5].data_ptr(), stream.cuda_stream), "ply")

    for _ in range(3):
        ingest()
    torch.cuda.synchronize(device)
    start.record(stream)
    for _ in range(steps):
        ingest()
    stop.record(stream)
    torch.cuda.synchronize(device)
    ply_ms = start.elapsed_time(stop) / steps
    ply_bytes = count * (4 * len(names) + 4 * (3 + 3 + 4 + 1 + width) + 8)
    # Hybrid composite of two layers.
    b, h, w = 64, 480, 640
    lay = [torch.rand((b, h, w, c), generator=gen).to(device) for c in (3, 1, 1, 3, 1, 1)]
    lay[2].mul_(10)
    lay[5].mul_(10)
    for _ in range(3):
        composite_gaussian_and_mesh(*lay)
    torch.cuda.synchronize(device)
    start.record(stream)
    for _ in range(steps):
        composite_gaussian_and_mesh(*lay)
    stop.record(stream)
    torch.cuda.synchronize(device)
    hyb_ms = start.elapsed_time(stop) / steps
    px = b * h * w
    hyb_bytes = px * (40 + 21)
    return {
        "ply_canonicalize": {"gaussians": count, "sh_degree": 3, "ms": round(ply_ms, 4),
                             "gaussians_per_s": round(count / (ply_ms / 1e3), 1),
                             "achieved_gbs": round(ply_bytes / (ply_ms / 1e3) / 1e9, 1),
                             "frac_of_hbm": round(ply_bytes / (ply_ms / 1e3) / 1e9 / peak, 4)},
        "hybrid_composite": {"pixels": px, "ms": round(hyb_ms, 4),
                             "mpix_per_s": round(px / (hyb_ms / 1e3) / 1e6, 1),
                             "achieved_gbs": round(hyb_bytes / (hyb_ms / 1e3) / 1e9, 1),
                             "frac_of_hbm": round(hyb_bytes / (hyb_ms / 1e3) / 1e9 / peak, 4)},
        "peak_gbs": peak, "peak_source": peak_source,
    }


def run_modes(args, device) -> dict:
    """The two alternative evaluation modes against the plain path, device
    time per frame with a fresh projection each frame (projection cache off):
    dense mode (tile_size=1, optical-thickness depth cutoff) on a deep scene
    (2M fairly opaque Gaussians, 32 cameras 320x240 orbiting inside the
    cloud's depth range, ~90% of tile keys hidden behind saturated pixels),
    and exact-ray evaluation on the batched 1M-Gaussian SH3 workload."""
    from vgr_b200 import CustomCudaBackend, RendererService
    from vgr_b200.workloads import batched_workload, orbit_cameras, synthetic_scene

    steps = max(args.mode_steps, 1)

    def frame_ms(scene, rig, **kw):
        backend = CustomCudaBackend(output_srgb=False, enable_projection_cache=False, **kw)
        svc = RendererService(backend, height=rig.height, width=rig.width, max_views=rig.viewmats.shape[0])
        svc.initialize(stage=None, device=device)
        svc.load_scene(1, **scene.to(device).as_kwargs())
        vm, k = rig.viewmats.to(device), rig.intrinsics.to(device)
        ids = torch.ones((vm.shape[0],), dtype=torch.int64, device=device)
        for _ in range(3):
            svc.render(vm, k, ids)
        torch.cuda.synchronize(device)
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record()
        for _ in range(steps):
            svc.render(vm, k, ids)
        stop.record()
        torch.cuda.synchronize(device)
        counters = backend.read_counters()
        out = {"ms": round(start.elapsed_time(stop) / steps, 3),
               "mpix_per_s": round(rig.viewmats.shape[0] * rig.height * rig.width
                                   / (start.elapsed_time(stop) / steps / 1e3) / 1e6, 1),
               "visible_records": counters["visible_gaussians"], "tile_keys": counters["tile_intersections"]}
        svc.shutdown()
        return out

    deep = synthetic_scene(2_000_000, seed=7, mean_half_extent=2.0, log_scale_mean=-3.0)
    deep.opacities.clamp_(min=0.5)
    deep_rig = orbit_cameras(args.mode_cameras or 32, seed=3, radius=6.0, width=320, height=240, focal=260.0)
    plain = frame_ms(deep, deep_rig, tile_size=16)
    dense = frame_ms(deep, deep_rig, tile_size=1)
    del deep
    scene, rig = batched_workload(cameras=args.mode_cameras or 64)
    screen = frame_ms(scene, rig, tile_size=16, sh_degree=3)
    ray = frame_ms(scene, rig, tile_size=16, sh_degree=3, ray_gaussian_evaluation=True)
    return {
        "dense_mode": {"workload": f"deep-2m-{deep_rig.viewmats.shape[0]}x320x240 (2M Gaussians, opacity >= 0.5)",
                       "plain_tile16": plain, "dense_tile1": dense,
                       "speedup": round(plain["ms"] / dense["ms"], 3)},
        "exact_ray": {"workload": f"batched-1m-sh3 ({rig.viewmats.shape[0]} cameras 640x480)", "screen_space": screen,
                      "exact_ray": ray, "ray_over_screen_time": round(ray["ms"] / screen["ms"], 3)},
        "steps": steps,
    }


def lidar_roofline(device, rays: int, trace_ms: float, trace_bytes: float, peak: float, peak_kind: str) -> dict:
    """The trace's binding resource is instruction issue (the scene and the
    hierarchy stay in L1/L2): warp instructions per ray from the recorded ncu
    capture x rays/s, against one issue per scheduler per cycle (4 per SM) at
    the B200's maximum SM clock.  The HBM figure is kept beside it."""
    rec = recorded_traffic(LIDAR_CONFIG["workload"])
    per_ray = rec.get("lidar_trace_kernel_warp_instructions_per_ray")
    sms = torch.cuda.get_device_properties(device).multi_processor_count
    peak_issue = sms * 4 * 1.965  # G warp instructions/s at 1965 MHz
    hbm = trace_bytes / (trace_ms / 1e3) / 1e9
    out = {"bound": "issue", "kernel": "lidar_trace_kernel", "unit": "G warp instr/s",
           "peak": round(peak_issue, 1), "peak_source": f"{sms} SMs x 4 schedulers x 1965 MHz (nominal maximum)",
           "warp_instructions_per_ray": per_ray, "instructions_source": rec.get("_source"),
           "issue_active_ncu": rec.get("_issue_active", {}).get("lidar_trace_kernel"),
           "hbm": {"achieved": round(hbm, 1), "peak": peak, "unit": "GB/s", "frac": round(hbm / peak, 4),
                   "peak_source": f"hbm_gbs of {peak_kind}", "algorithmic_bytes": int(trace_bytes)},
           "traffic": None}
    if per_ray:
        achieved = per_ray * rays / (trace_ms / 1e3) / 1e9
        out.update(achieved=round(achieved, 1), frac=round(achieved / peak_issue, 4))
    else:
        out.update(achieved=None, frac=None)
    return out


def run_lidar(args, device, world: int, with_cpu: bool) -> dict:
    """Gaussian LiDAR frames: rebuild the LBVH from moved means, then trace
    every ray of every sensor (first return)."""
    from vgr_b200 import workloads
    from vgr_b200.cuda_lidar_backend import CudaLidarBackend
    from vgr_b200.lidar_service import GaussianLidarService

    cfg = dict(LIDAR_CONFIG)
    if args.lidar_sensors:
        cfg["sensors"] = args.lidar_sensors
    work = workloads.lidar_workload(cfg["gaussians"], cfg["sensors"], cfg["beams"], cfg["azimuths"])
    sensors = cfg["sensors"]
    rays = work.ray_directions.shape[0]
    backend = CudaLidarBackend(far_plane_m=cfg["far_plane_m"], packet_size=cfg["packet"])
    service = GaussianLidarService(backend, max_sensors=sensors, max_rays=rays, returns=cfg["returns"])
    service.initialize(stage=None, device=device)
    scene = work.scene_kwargs(device)
    means = scene["means"]
    service.load_scene(0, **scene)
    moved = [lidar_moved_means(work.means, 100 + k).to(device) for k in range(2)]
    dirs = work.ray_directions.to(device)
    times = work.time_offsets_ns.to(device)
    poses = work.sensor_to_world.to(device)
    scene_ids = torch.zeros((sensors,), dtype=torch.int64, device=device)
    outputs = service.render_lidar(dirs, times, poses, scene_ids)

    def frame(k: int) -> None:
        means.copy_(moved[k % 2], non_blocking=True)
        backend.rebuild_scene(0)

    for k in range(max(args.warmup, 3)):
        frame(k)
        service.render_lidar(dirs, times, poses, scene_ids, outputs=outputs)
    torch.cuda.synchronize(device)
    counters0 = backend.check_errors()
    steps = max(args.lidar_steps, 1)
    stream = torch.cuda.current_stream(device)
    marks = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(steps)]
    barrier(world)
    torch.cuda.synchronize(device)
    for k in range(steps):
        marks[k][0].record(stream)
        frame(k + 1)
        marks[k][1].record(stream)
        service.render_lidar(dirs, times, poses, scene_ids, outputs=outputs)
        marks[k][2].record(stream)
    torch.cuda.synchronize(device)
    counters = backend.check_errors()
    total_ms = max_over_ranks(marks[0][0].elapsed_time(marks[-1][2]), world, device)
    build_ms = statistics.fmean(m[0].elapsed_time(m[1]) for m in marks)
    trace_ms = statistics.fmean(m[1].elapsed_time(m[2]) for m in marks)
    surfels = backend.surfel_count(0)
    traced = sensors * rays
    value = world * traced * steps / (total_ms / 1e3)

    # End to end: poses from pinned host memory, every output back to pinned
    # host memory, pipelined over two output sets (frame k's download on a
    # copy stream overlaps frame k+1's rebuild and trace).
    host_poses = work.sensor_to_world.pin_memory()
    sets = [outputs, {k: torch.empty_like(t) for k, t in outputs.items()}]
    host_sets = [{k: torch.empty(t.shape, dtype=t.dtype, pin_memory=True) for k, t in outputs.items()}
                 for _ in range(2)]
    d2h = sum(t.numel() * t.element_size() for t in host_sets[0].values())
    e_steps = max(2, min(steps, 5))
    copy_stream = torch.cuda.Stream(device)
    done = [None, None]
    torch.cuda.synchronize(device)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for k in range(e_steps):
        b = k % 2
        if done[b] is not None:
            stream.wait_event(done[b])
        poses.copy_(host_poses, non_blocking=True)
        frame(k)
        service.render_lidar(dirs, times, poses, scene_ids, outputs=sets[b])
        traced_ev = torch.cuda.Event()
        traced_ev.record(stream)
        copy_stream.wait_event(traced_ev)
        with torch.cuda.stream(copy_stream):
            for name, t in sets[b].items():
                host_sets[b][name].copy_(t, non_blocking=True)
        done[b] = torch.cuda.Event()
        done[b].record(copy_stream)
    for ev in done:
        if ev is not None:
            stream.wait_event(ev)
    e1.record(stream)
    torch.cuda.synchronize(device)
    e_ms = max_over_ranks(e0.elapsed_time(e1), world, device)

    leaves = -(-surfels // cfg["packet"])
    out_bytes = traced * (cfg["returns"] * (4 + 12 + 4 + 8 + 1 + 8) + 4)
    trace_bytes = traced * 12 + out_bytes + surfels * (80 + 8) + max(leaves - 1, 1) * 64
    peak, peak_kind = measured_peaks()
    result = {
        "metric": LIDAR_METRIC,
        "value": round(value, 1),
        "unit": "rays/s",
        "steps": steps,
        "ms_per_frame": round(total_ms / steps, 4),
        "build_ms": round(build_ms, 4),
        "trace_ms": round(trace_ms, 4),
        "config": {**cfg, "rays_per_frame": traced, "planar_surfels": surfels,
                   "returns_found_per_frame": (counters["returns"] - counters0["returns"]) // steps},
        "e2e": {"value": round(world * traced * e_steps / (e_ms / 1e3), 1), "unit": "rays/s",
                "h2d_bytes_per_step": host_poses.numel() * 4, "d2h_bytes_per_step": d2h, "steps": e_steps,
                "pipelined": "two output sets; frame k's download overlaps frame k+1"},
        "roofline": lidar_roofline(device, traced, trace_ms, trace_bytes, peak, peak_kind),
        "node_visits_per_ray": round((counters["node_visits"] - counters0["node_visits"]) / (steps * traced), 2),
        "leaf_tests_per_ray": round((counters["leaf_tests"] - counters0["leaf_tests"]) / (steps * traced), 2),
        "cpu_baseline": None,
    }
    service.shutdown()
    if with_cpu:
        cpu, threads, sample = lidar_cpu_sample(work)
        result["cpu_baseline"] = {"value": round(cpu, 1), "unit": "rays/s", "cores": threads, "kind": "port",
                                  "sample": sample}
    return result


# --------------------------------------------------------------------------- differentiable form
DIFF_METRIC = "fwd+bwd ms/iter, loss L2(RGB) + 0.1 L1(depth) vs a perturbed-scene target"


def run_differentiable(args, device, world: int) -> dict:
    """Differentiable form: 500k Gaussians (SH3) as raw parameters, 16 cameras
    of 512x512, loss L2(RGB) + 0.1 L1(depth) against images of a perturbed
    copy of the scene.  One step = training forward (activation, projection,
    tile sort, compositor with training outputs, capacity check) + loss +
    backward (compositor backward, per-Gaussian projection backward)."""
    from vgr_b200 import workloads
    from vgr_b200.differentiable import DifferentiableRenderer, photometric_loss

    from vgr_b200.distributed import allreduce_gradients

    rank = int(os.environ.get("RANK", "0"))
    # Data-parallel over cameras: every rank trains the same scene from its
    # own 16 cameras; the scene gradients are summed over ranks every step.
    work = workloads.training_workload(seed=13, camera_seed=15 + 7 * rank)
    rig = work.rig
    names = ("means", "log_scales", "rotations", "opacity_logits", "features")
    params = {k: v.to(device).requires_grad_(True) for k, v in work.params.items()}
    view = rig.viewmats.to(device)
    intr = rig.intrinsics.to(device)
    renderer = DifferentiableRenderer(height=rig.height, width=rig.width, sh_degree=3, device=device,
                                      capacity_check="deferred")
    target = [t.clone() for t in renderer.forward_native(*(work.targets[k].to(device) for k in names), view, intr)]
    t_rgb, t_depth = target[0], target[1]

    def step_with(r):
        def step() -> None:
            rgb, depth, _ = r.render(*(params[k] for k in names), view, intr)
            loss = photometric_loss(rgb, depth, t_rgb, t_depth, 0.1)
            loss.backward()
            if world > 1:
                allreduce_gradients([params[k].grad for k in names])
            for p in params.values():
                p.grad = None
        return step

    step = step_with(renderer)

    stream = torch.cuda.current_stream(device)
    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize(device)
    steps = max(args.diff_steps, 1)
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier(world)
    start.record(stream)
    for _ in range(steps):
        step()
    stop.record(stream)
    torch.cuda.synchronize(device)
    step_ms = max_over_ranks(start.elapsed_time(stop), world, device) / steps
    # Forward alone (the same training forward, no autograd).
    with torch.no_grad():
        detached = [params[k].detach() for k in names]
        for _ in range(3):
            renderer.forward_native(*detached, view, intr)
        torch.cuda.synchronize(device)
        start.record(stream)
        for _ in range(steps):
            renderer.forward_native(*detached, view, intr)
        stop.record(stream)
        torch.cuda.synchronize(device)
    fwd_ms = max_over_ranks(start.elapsed_time(stop), world, device) / steps
    # Backward kernels alone, from one forward (record clear + compositor
    # backward + projection backward), for the stage split.
    rgb, depth, alpha = renderer.forward_native(*detached, view, intr)
    g_rgb = torch.randn_like(rgb)
    g_depth = torch.randn_like(depth) * 0.1
    torch.cuda.synchronize(device)
    start.record(stream)
    for _ in range(steps):
        renderer.backward_native(renderer.frame, g_rgb, g_depth, None)
    stop.record(stream)
    torch.cuda.synchronize(device)
    bwd_ms = start.elapsed_time(stop) / steps
    # The same step under a list memory budget of a quarter of the frame's
    # lists: the forward renders camera chunks and the backward recomputes
    # each chunk's sorted lists.
    lc = renderer.last_counters
    full_lists = 24 * lc["tile_intersections"] + 96 * lc["visible_gaussians"] + \
        4 * work.params["means"].shape[0] * rig.viewmats.shape[0]
    budgeted = DifferentiableRenderer(height=rig.height, width=rig.width, sh_degree=3, device=device,
                                      list_budget_bytes=full_lists // 4, capacity_check="deferred")
    budget_step = step_with(budgeted)
    for _ in range(3):
        budget_step()
    torch.cuda.synchronize(device)
    start.record(stream)
    for _ in range(steps):
        budget_step()
    stop.record(stream)
    torch.cuda.synchronize(device)
    budget_ms = max_over_ranks(start.elapsed_time(stop), world, device) / steps
    budget_chunks = len(budgeted._pending["chunks"])
    pixels = rig.viewmats.shape[0] * rig.height * rig.width
    return {
        "metric": DIFF_METRIC,
        "value": round(step_ms, 3),
        "unit": "ms/iter",
        "higher_is_better": False,
        "steps": steps,
        "forward_ms": round(fwd_ms, 3),
        "backward_kernels_ms": round(bwd_ms, 3),
        "fwd_bwd_over_fwd": round(step_ms / fwd_ms, 3),
        "target_fwd_bwd_over_fwd": 2.5,
        "list_budget": {"budget_bytes": int(full_lists // 4), "full_lists_bytes": int(full_lists),
                        "camera_chunks": budget_chunks, "ms_per_iter": round(budget_ms, 3),
                        "mode": "lists beyond the budget are recomputed in the backward, not kept"},
        "gradients": "hand-written CUDA backward; float64 autograd + central-difference checks in tests",
        "parallelism": f"data-parallel x{world} (gradient all-reduce per step)" if world > 1 else "single-gpu",
        "capacity_check": "deferred: each forward's counters are read back asynchronously and checked "
                          "before its backward runs (an overflowed frame raises)",
        "loss": "fused photometric loss kernel (forward and gradient in one pass)",
        "config": {"workload": "train-500k-sh3-16x512", "gaussians": work.params["means"].shape[0],
                   "cameras": rig.viewmats.shape[0], "height": rig.height, "width": rig.width,
                   "pixels": pixels, "sh_degree": 3, "tile_size": renderer.tile_size,
                   "visible_records": renderer.last_counters.get("visible_gaussians"),
                   "tile_intersections": renderer.last_counters.get("tile_intersections")},
    }


def run_b200(args) -> None:
    world, rank, local = dist_setup()
    if not torch.cuda.is_available():
        raise RuntimeError("bench.py needs a CUDA device (the renderer has no CPU fallback)")
    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=device)

    from vgr_b200 import workloads

    frames = ragged_frames(args)
    work = workloads.ragged_workload(frames=frames, scale=args.ragged_scale)
    config = ragged_config(work, frames)
    head = run_ragged(args, device, world, rank, work)
    detail: dict = {"ragged": {k: v for k, v in head.items() if k in (
        "value", "ms", "tile", "persistent", "shape", "autotune_ms", "counters", "overflow", "split", "launches")}}
    detail["ragged"]["stage_ms"] = head["roofline"]["stage_ms"]
    detail["ragged"]["stage_frac_of_hbm"] = head["roofline"]["stage_frac_of_hbm"]

    plain = rgb = batched = diff = lidar = aux = modes = None
    if world == 1:
        if args.plain_steps > 0:
            plain = run_plain(args, device, work, head)
        for key in ("ragged", "holder", "backend", "last"):
            head.pop(key, None)
        torch.cuda.empty_cache()
        if args.rgb_steps > 0:
            rgb = run_ragged_rgb(args, device, work)
            torch.cuda.empty_cache()
        if args.batched_steps > 0:
            batched = run_batched(args, device)
            torch.cuda.empty_cache()
        if args.diff_steps > 0:
            diff = run_differentiable(args, device, world)
            torch.cuda.empty_cache()
        if args.lidar_steps > 0:
            lidar = run_lidar(args, device, world, with_cpu=not args.no_cpu_baseline)
            torch.cuda.empty_cache()
        if args.aux_steps > 0:
            aux = run_aux(args, device, world)
        if args.mode_steps > 0:
            modes = run_modes(args, device)

    cpu_baseline = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cams = cpu_sample_cameras(work, args.cpu_sample_cameras)
        value, _, threads, sample = time_ragged_cpu(work, cams, 1, 1)
        cpu_baseline = {"value": round(value, 3), "unit": UNIT, "cores": threads, "kind": "port",
                        "sample": sample}

    if rank == 0:
        detail.update({"plain_form": plain, "rgb_equation": rgb, "batched": batched, "differentiable": diff,
                       "lidar": lidar, "ingest_and_hybrid": aux, "modes": modes})
        line = {
            "metric": METRIC,
            "value": round(head["value"], 3),
            "unit": UNIT,
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": round(head["ms"], 4),
            "higher_is_better": True,
            "scaling": "strong",
            "vs_baseline": None,
            "dtype": "f32",
            "data": "synthetic",
            "config": config,
            "parallelism": ("single-gpu, one CUDA-graph submission per frame" if world == 1 else
                            f"ragged frame split over {world} ranks by estimated work, no data-path collective"),
            "e2e": head["e2e"],
            "gpu_launches": int(head["launches"]),
            "roofline": {k: v for k, v in head["roofline"].items() if k != "stage_frac_of_hbm"},
            "cpu_baseline": cpu_baseline,
            "clocks": head["clocks"],
            "capacity_overflow": head["overflow"],
            "autotune": {"tile": head["tile"], "persistent_compositor": head["persistent"],
                         "composite_shape": head["shape"]},
        }
        if plain is not None:
            line["plain_form"] = {k: plain[k] for k in ("value", "ms_per_frame", "calls_per_frame",
                                                        "rgb_max_abs_vs_ragged")}
            line["speedup_vs_plain"] = round(head["value"] / plain["value"], 3)
            line["target_speedup_vs_plain"] = 3.0
        if diff is not None:
            line["fwd_bwd"] = {"ms_per_iter": diff["value"], "forward_ms": diff["forward_ms"],
                               "ratio": diff["fwd_bwd_over_fwd"], "target_ratio": 2.5,
                               "workload": diff["config"]["workload"]}
        if batched is not None:
            line["batched"] = {"value": batched["value"], "ms_per_frame": batched["ms_per_frame"],
                               "composite_frac_of_hbm": batched["composite_frac_of_hbm"],
                               "workload": "batched-1m-sh3"}
        if rgb is not None:
            line["rgb_equation"] = {"ragged": rgb["value"],
                                    "batched": None if batched is None else batched["rgb_equation"]["value"],
                                    "note": "features[0..2] as linear RGB, the reference's equation"}
        if lidar is not None:
            line["lidar"] = {"value": lidar["value"], "unit": "rays/s", "ms_per_frame": lidar["ms_per_frame"],
                             "build_ms": lidar["build_ms"], "trace_ms": lidar["trace_ms"],
                             "e2e": lidar["e2e"]["value"], "workload": lidar["config"]["workload"]}
        text = json.dumps(detail, default=str)
        if args.detail:
            args.detail.parent.mkdir(parents=True, exist_ok=True)
            args.detail.write_text(text + "\n")
        print(text, file=sys.stderr, flush=True)
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


def reference_cuda_section(args, work) -> dict:
    """The reference's own CUDA path on this box (its Python classes on its
    CUDA build): the ragged frames (one call per resolution, features[0..2]
    as linear RGB), the batched frame, and the LiDAR frame."""
    from oracle import reference_cuda

    reason = reference_cuda.unavailable_reason()
    if reason is not None:
        return {"unavailable": reason}
    from vgr_b200 import workloads

    device = torch.device("cuda", 0)
    torch.cuda.set_device(device)
    sampler = ClockSampler(0)
    sampler.start()
    out: dict = {"equation": "features[0..2] as linear RGB (the reference's camera equation)"}
    frames = max(min(args.steps, 10), 2)
    ids = work.scene_ids.to(device)
    intr = work.intrinsics.to(device)
    poses = work.viewmats.to(device)
    ms, totals, _ = reference_cuda.camera_groups(work.scenes, group_by_resolution(work), intr, ids, poses,
                                                 device, frames)
    pixels = sum(h * w for h, w in zip(work.heights, work.widths))
    out["ragged"] = {"value": round(pixels / (ms / 1e3) / 1e6, 1), "ms_per_frame": round(ms, 3),
                     "calls_per_frame": 3, **totals}
    del poses
    torch.cuda.empty_cache()
    scene, rig = workloads.batched_workload()
    count = rig.viewmats.shape[0]
    ms, totals, _ = reference_cuda.camera_groups(
        [(0, scene)], {(rig.height, rig.width): list(range(count))}, rig.intrinsics.to(device),
        torch.zeros((count,), dtype=torch.int64, device=device), rig.viewmats.to(device)[None], device, frames)
    out["batched"] = {"value": round(count * rig.height * rig.width / (ms / 1e3) / 1e6, 1),
                      "ms_per_frame": round(ms, 3), **totals}
    del scene, rig
    torch.cuda.empty_cache()
    if args.lidar_steps > 0:
        cfg = LIDAR_CONFIG
        lw = workloads.lidar_workload(cfg["gaussians"], cfg["sensors"], cfg["beams"], cfg["azimuths"])
        moved = [lidar_moved_means(lw.means, 100 + k).to(device) for k in range(2)]
        ms, found = reference_cuda.lidar_frames(lw, device, max(args.lidar_steps, 1), moved,
                                                cfg["far_plane_m"], cfg["packet"])
        rays = lw.ray_directions.shape[0] * cfg["sensors"]
        out["lidar"] = {"value": round(rays / (ms / 1e3), 1), "unit": "rays/s", "ms_per_frame": round(ms, 3),
                        "returns_found": found}
    out["clocks"] = sampler.stop()
    return out


def run_reference(args) -> None:
    world, rank, _ = dist_setup()
    if rank != 0:
        return
    from vgr_b200 import workloads

    frames = ragged_frames(args)
    work = workloads.ragged_workload(frames=frames, scale=args.ragged_scale)
    config = ragged_config(work, frames)
    cams = cpu_sample_cameras(work, args.cpu_sample_cameras)
    steps = max(args.steps, 1)
    value, seconds, threads, sample = time_ragged_cpu(work, cams, steps, args.warmup)
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": round(value, 3),
        "unit": UNIT,
        "n_gpus": args.gpus,
        "steps": steps,
        "warmup": args.warmup,
        "ms_per_step": round(seconds * 1e3 / steps, 3),
        "higher_is_better": True,
        "scaling": "strong",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic",
        "config": config,
        "cpu_baseline": {"value": round(value, 3), "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": sample},
        "e2e": {"value": round(value, 3), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "the reference has no CPU renderer; its CPU path is the oracle's restatement of its equation",
    }
    if args.lidar_steps > 0:
        from vgr_b200 import workloads as wl

        cfg = LIDAR_CONFIG
        lw = wl.lidar_workload(cfg["gaussians"], cfg["sensors"], cfg["beams"], cfg["azimuths"])
        rays_per_s, lidar_threads, lidar_sample = lidar_cpu_sample(lw)
        line["lidar"] = {"value": round(rays_per_s, 1), "unit": "rays/s", "cores": lidar_threads,
                         "kind": "port", "sample": lidar_sample}
    if not args.no_reference_cuda:
        try:
            line["reference_cuda"] = reference_cuda_section(args, work)
        except Exception as error:  # report, do not fail the CPU arm
            line["reference_cuda"] = {"unavailable": f"{type(error).__name__}: {error}"[:300]}
    print(json.dumps(line), flush=True)


def main() -> None:
    args = parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
