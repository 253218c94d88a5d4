"""Seeded synthetic scenes and camera rigs of the benchmark workloads.

No public dataset is used by the benchmark: scenes and cameras are drawn from
the stated distributions with a CPU torch.Generator, so the CUDA path and the
CPU oracle see bit-identical inputs.

Workloads (all float32):
  plain-10k-256   10,000 Gaussians, means U[-1,1]^3, log-scales N(-4,0.5),
                  quaternions normalised N(0,I4) (WXYZ), opacity
                  sigmoid(N(0,1)), RGB U[0,1], semantic U{0..15}; one pinhole
                  256x256 camera, fx=fy=256, cx=cy=128, at (0,0,-3) looking at
                  the origin.
  batched-1m-sh3  1,000,000 Gaussians with means U[-5,5]^3 and degree-3
                  spherical harmonics (48 coefficients: DC from U[0,1] colour,
                  the rest N(0,0.2)); 64 pinhole 640x480 cameras, fx=fy=525,
                  on a radius-8 orbit at height 1.5 with +-5 deg yaw jitter,
                  all looking at the origin.
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import torch

SH_C0 = 0.28209479177387814


@dataclass
class SceneTensors:
    means: torch.Tensor
    scales: torch.Tensor
    rotations: torch.Tensor
    opacities: torch.Tensor
    features: torch.Tensor
    semantic_ids: torch.Tensor

    def to(self, device: torch.device | str) -> "SceneTensors":
        return SceneTensors(
            **{name: getattr(self, name).to(device).contiguous() for name in self.__dataclass_fields__}
        )

    def as_kwargs(self) -> dict[str, torch.Tensor]:
        return {name: getattr(self, name) for name in self.__dataclass_fields__}


@dataclass
class CameraRig:
    viewmats: torch.Tensor  # [B,4,4] world -> OpenCV camera
    intrinsics: torch.Tensor  # [B,3,3]
    height: int
    width: int

    def to(self, device: torch.device | str) -> "CameraRig":
        return CameraRig(
            self.viewmats.to(device).contiguous(),
            self.intrinsics.to(device).contiguous(),
            self.height,
            self.width,
        )


def synthetic_scene(
    count: int,
    *,
    seed: int,
    mean_half_extent: float = 1.0,
    log_scale_mean: float = -4.0,
    log_scale_std: float = 0.5,
    sh_degree: int | None = None,
    semantic_classes: int = 16,
) -> SceneTensors:
    """Scene drawn with a CPU generator (see module docstring for the laws)."""
    gen = torch.Generator().manual_seed(seed)
    means = (torch.rand((count, 3), generator=gen) * 2.0 - 1.0) * mean_half_extent
    scales = torch.exp(torch.randn((count, 3), generator=gen) * log_scale_std + log_scale_mean)
    quats = torch.randn((count, 4), generator=gen)
    quats = quats / quats.norm(dim=1, keepdim=True).clamp_min(1e-12)
    opacities = torch.sigmoid(torch.randn((count,), generator=gen))
    rgb = torch.rand((count, 3), generator=gen)
    if sh_degree is None:
        features = rgb
    else:
        k = (sh_degree + 1) ** 2
        coeffs = torch.randn((count, k, 3), generator=gen) * 0.2
        coeffs[:, 0, :] = (rgb - 0.5) / SH_C0
        features = coeffs.reshape(count, k * 3)
    semantic_ids = torch.randint(0, semantic_classes, (count,), generator=gen, dtype=torch.int32)
    return SceneTensors(
        means=means.float().contiguous(),
        scales=scales.float().contiguous(),
        rotations=quats.float().contiguous(),
        opacities=opacities.float().contiguous(),
        features=features.float().contiguous(),
        semantic_ids=semantic_ids.to(torch.int64).contiguous(),
    )


def look_at_viewmats(eyes: torch.Tensor, targets: torch.Tensor, up=(0.0, 1.0, 0.0)) -> torch.Tensor:
    """OpenCV world->camera matrices (x right, y down, z forward), float64 math."""
    eyes = eyes.double()
    targets = targets.double()
    up_t = torch.tensor(up, dtype=torch.float64).expand_as(eyes)
    z = targets - eyes
    z = z / z.norm(dim=1, keepdim=True)
    y_hint = -up_t
    x = torch.linalg.cross(y_hint, z, dim=1)
    x = x / x.norm(dim=1, keepdim=True)
    y = torch.linalg.cross(z, x, dim=1)
    rot = torch.stack((x, y, z), dim=1)
    trans = -(rot @ eyes.unsqueeze(-1)).squeeze(-1)
    view = torch.zeros((eyes.shape[0], 4, 4), dtype=torch.float64)
    view[:, :3, :3] = rot
    view[:, :3, 3] = trans
    view[:, 3, 3] = 1.0
    return view.float().contiguous()


def pinhole(batch: int, fx: float, fy: float, cx: float, cy: float) -> torch.Tensor:
    k = torch.zeros((batch, 3, 3), dtype=torch.float32)
    k[:, 0, 0] = fx
    k[:, 1, 1] = fy
    k[:, 0, 2] = cx
    k[:, 1, 2] = cy
    k[:, 2, 2] = 1.0
    return k


def plain_camera(height: int = 256, width: int = 256, focal: float = 256.0, distance: float = 3.0) -> CameraRig:
    eyes = torch.tensor([[0.0, 0.0, -distance]])
    view = look_at_viewmats(eyes, torch.zeros((1, 3)))
    return CameraRig(view, pinhole(1, focal, focal, width / 2.0, height / 2.0), height, width)


def orbit_cameras(
    count: int,
    *,
    seed: int,
    radius: float = 8.0,
    height_offset: float = 1.5,
    yaw_jitter_deg: float = 5.0,
    width: int = 640,
    height: int = 480,
    focal: float = 525.0,
) -> CameraRig:
    gen = torch.Generator().manual_seed(seed)
    base = torch.arange(count, dtype=torch.float64) * (2.0 * math.pi / count)
    jitter = (torch.rand((count,), generator=gen, dtype=torch.float64) * 2.0 - 1.0) * math.radians(yaw_jitter_deg)
    yaw = base + jitter
    eyes = torch.stack((radius * torch.cos(yaw), torch.full_like(yaw, height_offset), radius * torch.sin(yaw)), dim=1)
    view = look_at_viewmats(eyes, torch.zeros((count, 3), dtype=torch.float64))
    return CameraRig(view, pinhole(count, focal, focal, width / 2.0, height / 2.0), height, width)


@dataclass
class LidarWorkload:
    means: torch.Tensor
    scales: torch.Tensor
    rotations: torch.Tensor
    opacities: torch.Tensor
    semantic_ids: torch.Tensor
    reflectivity: torch.Tensor
    ray_directions: torch.Tensor  # [R,3] sensor frame
    time_offsets_ns: torch.Tensor  # [R] int64
    sensor_to_world: torch.Tensor  # [B,4,4]

    def scene_kwargs(self, device) -> dict[str, torch.Tensor]:
        return {
            name: getattr(self, name).to(device).contiguous()
            for name in ("means", "scales", "rotations", "opacities", "semantic_ids", "reflectivity")
        }


def spinning_lidar_rays(beams: int = 128, azimuths: int = 2048, low_deg: float = -25.0,
                        high_deg: float = 15.0) -> tuple[torch.Tensor, torch.Tensor]:
    """Unit rays of a spinning LiDAR: beams evenly spaced in elevation, azimuth-major order."""
    elev = torch.linspace(math.radians(low_deg), math.radians(high_deg), beams, dtype=torch.float64)
    azim = torch.arange(azimuths, dtype=torch.float64) * (2.0 * math.pi / azimuths)
    a, e = torch.meshgrid(azim, elev, indexing="ij")
    dirs = torch.stack((torch.cos(e) * torch.cos(a), torch.cos(e) * torch.sin(a), torch.sin(e)), dim=-1)
    dirs = dirs.reshape(-1, 3)
    dirs = dirs / dirs.norm(dim=1, keepdim=True)
    # One revolution in 100 ms, azimuth-major.
    times = (torch.arange(azimuths, dtype=torch.int64) * (100_000_000 // azimuths)).repeat_interleave(beams)
    return dirs.float().contiguous(), times.contiguous()


def lidar_workload(gaussians: int = 2_000_000, sensors: int = 64, beams: int = 128,
                   azimuths: int = 2048, seed: int = 5) -> LidarWorkload:
    """Gaussian LiDAR tracing: Gaussians in a 40 x 40 x 6 m box, log-scales
    N(-3, 0.5), reflectivity U[0,1], semantic U{0..15}; spinning sensors of
    `beams` x `azimuths` rays at random positions 1-2 m above the floor."""
    gen = torch.Generator().manual_seed(seed)
    lo = torch.tensor([-20.0, -20.0, 0.0], dtype=torch.float64)
    ext = torch.tensor([40.0, 40.0, 6.0], dtype=torch.float64)
    means = lo + torch.rand((gaussians, 3), generator=gen, dtype=torch.float64) * ext
    scales = torch.exp(torch.randn((gaussians, 3), generator=gen) * 0.5 - 3.0)
    quats = torch.randn((gaussians, 4), generator=gen)
    quats = quats / quats.norm(dim=1, keepdim=True)
    opacities = torch.sigmoid(torch.randn((gaussians,), generator=gen))
    reflectivity = torch.rand((gaussians,), generator=gen)
    semantic = torch.randint(0, 16, (gaussians,), generator=gen, dtype=torch.int64)
    dirs, times = spinning_lidar_rays(beams, azimuths)
    pos = torch.stack(
        (
            torch.rand((sensors,), generator=gen, dtype=torch.float64) * 36.0 - 18.0,
            torch.rand((sensors,), generator=gen, dtype=torch.float64) * 36.0 - 18.0,
            1.0 + torch.rand((sensors,), generator=gen, dtype=torch.float64),
        ),
        dim=1,
    )
    yaw = torch.rand((sensors,), generator=gen, dtype=torch.float64) * 2.0 * math.pi
    xform = torch.zeros((sensors, 4, 4), dtype=torch.float64)
    xform[:, 0, 0] = torch.cos(yaw)
    xform[:, 0, 1] = -torch.sin(yaw)
    xform[:, 1, 0] = torch.sin(yaw)
    xform[:, 1, 1] = torch.cos(yaw)
    xform[:, 2, 2] = 1.0
    xform[:, :3, 3] = pos
    xform[:, 3, 3] = 1.0
    return LidarWorkload(
        means=means.float().contiguous(),
        scales=scales.float().contiguous(),
        rotations=quats.float().contiguous(),
        opacities=opacities.float().contiguous(),
        semantic_ids=semantic.contiguous(),
        reflectivity=reflectivity.float().contiguous(),
        ray_directions=dirs,
        time_offsets_ns=times,
        sensor_to_world=xform.float().contiguous(),
    )


def plain_workload() -> tuple[SceneTensors, CameraRig]:
    """Plain single-camera forward render: 10k Gaussians, 256x256."""
    return synthetic_scene(10_000, seed=0), plain_camera()


def batched_workload(gaussians: int = 1_000_000, cameras: int = 64) -> tuple[SceneTensors, CameraRig]:
    """Batched forward render: 1M Gaussians SH degree 3, 64 cameras 640x480."""
    scene = synthetic_scene(gaussians, seed=1, mean_half_extent=5.0, sh_degree=3)
    return scene, orbit_cameras(cameras, seed=2)


# --------------------------------------------------------------------------- ragged batch
RAGGED_SCENE_SIZES = (100_000, 250_000, 500_000, 750_000, 1_000_000, 1_500_000, 2_000_000, 3_000_000)
RAGGED_CAMERAS_PER_SCENE = (32, 64, 96, 128, 128, 160, 160, 256)
RAGGED_RESOLUTIONS = ((128, 128), (120, 160), (240, 320))  # (height, width)


@dataclass
class RaggedWorkload:
    scenes: list[tuple[int, SceneTensors]]
    scene_ids: torch.Tensor  # [B] int64, cameras grouped by scene
    heights: list[int]
    widths: list[int]
    viewmats: torch.Tensor  # [F, B, 4, 4] per-frame world -> OpenCV camera
    intrinsics: torch.Tensor  # [B, 3, 3]


def ragged_workload(frames: int = 100, *, seed: int = 7, scale: float = 1.0) -> RaggedWorkload:
    """Ragged batch: eight scenes of 100k..3M Gaussians (distributions of the
    batched workload: means U[-5,5]^3, SH degree 3), 1,024 cameras split
    32..256 per scene, each at a resolution drawn from 128x128 / 160x120 /
    320x240, fx = fy = 0.75 W; poses at random positions inside the scene
    bounds, yaw U[0, 2pi), pitch U[-15, 15] deg; each frame moves every
    camera by N(0, 0.01) per axis and turns it by N(0, 0.5 deg).  ``scale``
    shrinks scene sizes and camera counts for small checks."""
    gen = torch.Generator().manual_seed(seed)
    scenes = []
    counts = []
    for k, (size, cams) in enumerate(zip(RAGGED_SCENE_SIZES, RAGGED_CAMERAS_PER_SCENE)):
        scenes.append((k, synthetic_scene(max(int(size * scale), 1), seed=100 + k, mean_half_extent=5.0,
                                          sh_degree=3)))
        counts.append(max(int(round(cams * scale)), 1))
    batch = sum(counts)
    scene_ids = torch.cat([torch.full((c,), k, dtype=torch.int64) for k, c in enumerate(counts)])
    choice = torch.randint(0, len(RAGGED_RESOLUTIONS), (batch,), generator=gen)
    heights = [RAGGED_RESOLUTIONS[int(i)][0] for i in choice]
    widths = [RAGGED_RESOLUTIONS[int(i)][1] for i in choice]
    pos = (torch.rand((batch, 3), generator=gen, dtype=torch.float64) * 2.0 - 1.0) * 5.0
    yaw = torch.rand((batch,), generator=gen, dtype=torch.float64) * 2.0 * math.pi
    pitch = (torch.rand((batch,), generator=gen, dtype=torch.float64) * 2.0 - 1.0) * math.radians(15.0)
    views = []
    for _ in range(frames):
        direction = torch.stack(
            (torch.cos(pitch) * torch.cos(yaw), torch.sin(pitch), torch.cos(pitch) * torch.sin(yaw)), dim=1
        )
        views.append(look_at_viewmats(pos, pos + direction))
        pos = pos + torch.randn((batch, 3), generator=gen, dtype=torch.float64) * 0.01
        yaw = yaw + torch.randn((batch,), generator=gen, dtype=torch.float64) * math.radians(0.5)
    intr = torch.zeros((batch, 3, 3), dtype=torch.float32)
    for c in range(batch):
        w, h = widths[c], heights[c]
        intr[c] = pinhole(1, 0.75 * w, 0.75 * w, w / 2.0, h / 2.0)[0]
    return RaggedWorkload(scenes, scene_ids, heights, widths, torch.stack(views).contiguous(), intr)


# --------------------------------------------------------------------------- differentiable form
@dataclass
class TrainingWorkload:
    params: dict[str, torch.Tensor]   # means, log_scales, rotations, opacity_logits, features
    targets: dict[str, torch.Tensor]  # the target scene's parameters (perturbed copy)
    rig: CameraRig


def training_workload(gaussians: int = 500_000, cameras: int = 16, size: int = 512, *,
                      seed: int = 13, camera_seed: int | None = None) -> TrainingWorkload:
    """Differentiable-form workload: a 500k-Gaussian SH3 scene (the batched
    scene's laws) as raw parameters, 16 orbit cameras of 512x512 (focal 420),
    and a target scene = means + N(0, 0.01), SH coefficients + N(0, 0.05)."""
    scene = synthetic_scene(gaussians, seed=seed, mean_half_extent=5.0, sh_degree=3)
    params = {
        "means": scene.means,
        "log_scales": torch.log(scene.scales),
        "rotations": scene.rotations,
        "opacity_logits": torch.logit(scene.opacities.double(), eps=1e-6).float(),
        "features": scene.features,
    }
    gen = torch.Generator().manual_seed(seed + 1)
    targets = dict(params)
    targets["means"] = (params["means"] + torch.randn(params["means"].shape, generator=gen) * 0.01).contiguous()
    targets["features"] = (params["features"] + torch.randn(params["features"].shape, generator=gen) * 0.05).contiguous()
    rig = orbit_cameras(cameras, seed=seed + 2 if camera_seed is None else camera_seed,
                        width=size, height=size, focal=420.0)
    return TrainingWorkload(params=params, targets=targets, rig=rig)
