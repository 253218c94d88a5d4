"""CUDA Gaussian LiDAR vs the reference oracle's golden vectors and the CPU oracle.

Tolerances are the path's: range (and hence position) within 1e-4 m,
intensity within 1e-4, valid / semantic / return counts exact.  The kernels
compute in float32 (cluster sums in float64) and the oracles in float64.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from golden import lidar_cases
from oracle import lidar as ol
from vgr_b200.cuda_lidar_backend import CudaLidarBackend
from vgr_b200.lidar_service import GaussianLidarService
from vgr_b200.workloads import lidar_workload

pytestmark = pytest.mark.gpu


def _f32(a):
    return torch.as_tensor(np.asarray(a), dtype=torch.float32).contiguous()


def _gpu_render(case, packet=8, **backend_kwargs):
    device = torch.device("cuda")
    sensors = case["sensors"]
    batch = sensors.shape[0]
    rays = case["rays"].shape[0]
    backend = CudaLidarBackend(packet_size=packet, **backend_kwargs)
    service = GaussianLidarService(backend, max_sensors=batch, max_rays=rays, returns=case["kwargs"]["returns"])
    service.initialize(stage=None, device=device)
    for sid, scene in case["scenes"].items():
        service.load_scene(
            sid,
            means=_f32(scene["means"]).to(device),
            scales=_f32(scene["scales"]).to(device),
            rotations=_f32(scene["rotations"]).to(device),
            opacities=_f32(scene["opacities"]).to(device),
            semantic_ids=torch.as_tensor(scene["semantic_ids"], dtype=torch.int64).to(device),
            reflectivity=None if scene["reflectivity"] is None else _f32(scene["reflectivity"]).to(device),
            surface_confidence=None
            if scene["surface_confidence"] is None
            else _f32(scene["surface_confidence"]).to(device),
        )
    kwargs = {}
    if "scene_to_world" in case["kwargs"]:
        kwargs["scene_to_world"] = _f32(case["kwargs"]["scene_to_world"]).to(device)
    if "active_sensor_ids" in case["kwargs"]:
        kwargs["active_sensor_ids"] = torch.as_tensor(case["kwargs"]["active_sensor_ids"], dtype=torch.int64).to(device)
    out = service.render_lidar(
        _f32(case["rays"]).to(device),
        torch.as_tensor(case["times"], dtype=torch.int64).to(device),
        _f32(sensors).to(device),
        torch.as_tensor(case["scene_ids"], dtype=torch.int64).to(device),
        **kwargs,
    )
    service.synchronize()
    counters = backend.check_errors()
    return {k: v.cpu().numpy() for k, v in out.items()}, counters


def _compare(got, want, atol=1e-4):
    for key in ("valid", "semantic_id", "return_count", "time_offset_ns"):
        np.testing.assert_array_equal(got[key], np.asarray(want[key]).astype(got[key].dtype), err_msg=key)
    valid = np.asarray(want["valid"]).astype(bool)
    np.testing.assert_allclose(got["range_m"][valid], want["range_m"][valid], rtol=0, atol=atol)
    assert np.all(np.isinf(got["range_m"][~valid]))
    np.testing.assert_allclose(got["intensity"][valid], want["intensity"][valid], rtol=0, atol=atol)
    np.testing.assert_allclose(got["position_world_m"][valid], want["position_world_m"][valid], rtol=0, atol=atol)
    assert np.all(got["position_world_m"][~valid] == 0)


@pytest.mark.parametrize("name", lidar_cases.names())
@pytest.mark.parametrize("packet", [8, 16])
def test_lidar_matches_reference_golden(name, packet):
    case = lidar_cases.load(name)
    got, counters = _gpu_render(case, packet)
    _compare(got, case["expected"])
    assert counters["returns"] == int(np.asarray(case["expected"]["valid"]).sum())
    assert counters["calls_started"] == counters["calls_completed"] == 1


def test_lidar_matches_cpu_oracle_on_random_scene():
    work = lidar_workload(gaussians=20_000, sensors=3, beams=16, azimuths=64, seed=11)
    # Shrink the box so most rays hit something.
    means = work.means * torch.tensor([0.15, 0.15, 0.5])
    scene = {
        "means": means.double().numpy(),
        "scales": work.scales.double().numpy(),
        "rotations": work.rotations.double().numpy(),
        "opacities": work.opacities.double().numpy(),
        "semantic_ids": work.semantic_ids.numpy(),
        "reflectivity": work.reflectivity.double().numpy(),
        "surface_confidence": None,
    }
    sensors = work.sensor_to_world.double().numpy().copy()
    sensors[:, :3, 3] *= np.array([0.15, 0.15, 1.0])
    case = {
        "scenes": {3: scene},
        "rays": work.ray_directions.double().numpy(),
        "times": work.time_offsets_ns.numpy(),
        "sensors": sensors,
        "scene_ids": np.array([3, 3, 3]),
        "kwargs": {"returns": 2},
    }
    want = ol.render(case["scenes"], case["rays"], case["times"], case["sensors"], case["scene_ids"], returns=2)
    got, counters = _gpu_render(case)
    assert counters["returns"] > 50
    # Float32 traversal vs float64 oracle: allow rare boundary flips but not more.
    agree = (got["valid"] == want["valid"]).mean()
    assert agree >= 0.999, agree
    both = got["valid"] & want["valid"]
    same_first = both[..., 0]
    np.testing.assert_allclose(got["range_m"][..., 0][same_first], want["range_m"][..., 0][same_first], rtol=0, atol=1e-4)
    assert (got["semantic_id"][both] == want["semantic_id"][both]).mean() >= 0.999


def test_lidar_rebuild_after_revision_matches_oracle():
    case = lidar_cases.load("random_2027")
    device = torch.device("cuda")
    scene = case["scenes"][5]
    batch = case["sensors"].shape[0]
    backend = CudaLidarBackend()
    service = GaussianLidarService(backend, max_sensors=batch, max_rays=case["rays"].shape[0], returns=2)
    service.initialize(stage=None, device=device)
    means = _f32(scene["means"]).to(device)
    service.load_scene(
        5,
        means=means,
        scales=_f32(scene["scales"]).to(device),
        rotations=_f32(scene["rotations"]).to(device),
        opacities=_f32(scene["opacities"]).to(device),
        semantic_ids=torch.as_tensor(scene["semantic_ids"]).to(device),
        reflectivity=_f32(scene["reflectivity"]).to(device),
        surface_confidence=_f32(scene["surface_confidence"]).to(device),
    )
    shift = np.zeros_like(scene["means"])
    shift[::7, 0] = 0.5
    means.add_(_f32(shift).to(device))
    service.revise_scene(5, revision=1)
    out = service.render_lidar(
        _f32(case["rays"]).to(device),
        torch.as_tensor(case["times"]).to(device),
        _f32(case["sensors"]).to(device),
        torch.as_tensor(case["scene_ids"]).to(device),
    )
    service.synchronize()
    moved = dict(scene)
    moved["means"] = means.double().cpu().numpy()
    want = ol.render({5: moved}, case["rays"], case["times"], case["sensors"], case["scene_ids"], returns=2)
    got = {k: v.cpu().numpy() for k, v in out.items()}
    _compare(got, want)


def test_lidar_invalid_inputs_are_counted_not_faulted():
    case = lidar_cases.load("two_returns")
    device = torch.device("cuda")
    backend = CudaLidarBackend()
    service = GaussianLidarService(backend, max_sensors=3, max_rays=2, returns=1)
    service.initialize(stage=None, device=device)
    scene = case["scenes"][4]
    service.load_scene(
        4,
        means=_f32(scene["means"]).to(device),
        scales=_f32(scene["scales"]).to(device),
        rotations=_f32(scene["rotations"]).to(device),
        opacities=_f32(scene["opacities"]).to(device),
        semantic_ids=torch.as_tensor(scene["semantic_ids"]).to(device),
    )
    rays = _f32([[1.0, 0.0, 0.0], [0.0, 2.0, 0.0]]).to(device)  # second ray not unit
    sensors = torch.eye(4, device=device).repeat(3, 1, 1).contiguous()
    scene_ids = torch.tensor([4, 99, 4], device=device)  # 99 unregistered
    out = service.render_lidar(
        rays, torch.zeros(2, dtype=torch.int64, device=device), sensors, scene_ids,
        active_sensor_ids=torch.tensor([0, 1], device=device),
    )
    service.synchronize()
    counters = backend.read_counters()
    # Direction validity is checked before the scene lookup (reference order).
    assert counters["invalid_directions"] == 2
    assert counters["invalid_scene_ids"] == 1
    assert bool(out["valid"][0, 0, 0]) and not out["valid"][2].any()
    assert torch.isinf(out["range_m"][1]).all()


@pytest.mark.parametrize("order", ["identity", "reversed", "random"])
def test_lidar_trace_order_does_not_change_returns(monkeypatch, order):
    # The backend traces rays in the Morton order of their directions
    # (RayOrder); any other permutation gives the same returns, and outputs
    # stay indexed by ray.
    import vgr_b200.cuda_lidar_backend as clb

    case = lidar_cases.load("random_2027")
    morton, _ = _gpu_render(case)

    def make(directions):
        n = directions.shape[0]
        if order == "identity":
            return torch.arange(n, dtype=torch.int32, device=directions.device)
        if order == "reversed":
            return torch.arange(n - 1, -1, -1, dtype=torch.int32, device=directions.device)
        gen = torch.Generator().manual_seed(11)
        return torch.randperm(n, generator=gen).to(torch.int32).to(directions.device)

    monkeypatch.setattr(clb.RayOrder, "__call__", lambda self, directions: make(directions))
    got, _ = _gpu_render(case)
    for key in ("valid", "semantic_id", "return_count", "time_offset_ns"):
        np.testing.assert_array_equal(got[key], morton[key], err_msg=key)
    valid = morton["valid"].astype(bool)
    for key in ("range_m", "intensity", "position_world_m"):
        np.testing.assert_allclose(got[key][valid], morton[key][valid], rtol=0, atol=1e-6, err_msg=key)


def test_lidar_ray_order_outside_the_rays_is_counted_not_faulted(monkeypatch):
    import vgr_b200.cuda_lidar_backend as clb

    case = lidar_cases.load("random_2027")
    rays = case["rays"].shape[0]
    bad = torch.arange(rays, dtype=torch.int32)
    bad[0] = rays  # past the end: that work item traces nothing, ray 0 stays cleared
    monkeypatch.setattr(clb.RayOrder, "__call__", lambda self, directions: bad.to(directions.device))
    with pytest.raises(clb.LidarTraversalError, match="invalid_directions"):
        _gpu_render(case)


def test_lidar_ray_order_is_a_permutation_in_compact_patches():
    # vgr_lidar_ray_order on a spinning LiDAR's 2048 x 128 grid (azimuth-major):
    # a permutation whose warps of 32 rays each span a small patch of azimuth
    # and beam indices.
    from vgr_b200.cuda_lidar_backend import RayOrder
    from vgr_b200.workloads import spinning_lidar_rays

    dirs, _ = spinning_lidar_rays(128, 2048)
    order = RayOrder()(dirs.cuda()).cpu().numpy()
    np.testing.assert_array_equal(np.sort(order), np.arange(dirs.shape[0]))
    az, beam = order // 128, order % 128
    az_span = np.ptp(az.reshape(-1, 32), axis=1)
    beam_span = np.ptp(beam.reshape(-1, 32), axis=1)
    # Outside the azimuth seam a warp typically covers 8 azimuths x 4 beams
    # (1.4 x 1.3 degrees) and rarely more than 24 x 8; the given order spans
    # 1 x 32.
    inner = az_span < 1024
    assert inner.mean() > 0.99
    assert np.median(az_span[inner]) <= 10 and np.median(beam_span[inner]) <= 5
    assert np.percentile(az_span[inner], 99) <= 24 and np.percentile(beam_span[inner], 99) <= 8
