"""The reference's own service and backend classes, unchanged, rendering on
this library's drop-in native modules.

The reference lets a backend be given its native module
(``CustomCudaBackend(native_module=...)``, cuda_backend.py:123-124,266,
317-318; ``CudaLidarBackend(native_module=...)``, cuda_lidar_backend.py:
79-80,118,132-133).  These tests construct the reference's
``RendererService``/``CustomCudaBackend`` and ``GaussianLidarService``/
``CudaLidarBackend`` with ``vgr_b200.native_module`` and
``vgr_b200.lidar_native_module`` injected, so the reference's workspace
planner, capacity grow/retry loop, chunked submission, projection cache and
LiDAR build/pack/trace sequence all run against this library, and compare
the results with the CPU oracle (camera, bit for bit) and with the golden
vectors of the reference's LiDAR oracle (within 1e-4 m).

The reference's Python package is pure Python (its own extensions are built
only on first use, which never happens here).  It is imported from
``baseline/_ref`` (``python -m pip install --no-deps --target baseline/_ref
<reference checkout>``) or from the import path; without it these tests are
skipped with that reason.  ``plyfile`` (imported by the package's PLY loader,
unused here) is stubbed when absent.
"""

from __future__ import annotations

import math
import sys
import types
from pathlib import Path

import numpy as np
import pytest
import torch

from golden import lidar_cases
from helpers import assert_bitwise_equal, render_oracle
from vgr_b200 import native_module
from vgr_b200.lidar_native_module import load_lidar_extension
from vgr_b200.workloads import CameraRig, orbit_cameras, plain_workload, synthetic_scene

pytestmark = pytest.mark.gpu

_BASELINE = Path(__file__).resolve().parents[1] / "baseline" / "_ref"


def _reference_package():
    if _BASELINE.is_dir() and str(_BASELINE) not in sys.path:
        sys.path.append(str(_BASELINE))
    if "plyfile" not in sys.modules:
        try:
            import plyfile  # noqa: F401
        except ImportError:
            stub = types.ModuleType("plyfile")
            stub.PlyData = stub.PlyElement = object
            sys.modules["plyfile"] = stub
    try:
        import isaacsim_gaussian_renderer as ref
        from isaacsim_gaussian_renderer.cuda_backend import CustomCudaBackend
        from isaacsim_gaussian_renderer.cuda_lidar_backend import CudaLidarBackend
    except ImportError as error:
        pytest.skip(f"the reference's Python package is not installed under baseline/_ref ({error})")
    return ref, CustomCudaBackend, CudaLidarBackend


def _reference_camera_service(rig, scenes, **backend_kwargs):
    ref, CustomCudaBackend, _ = _reference_package()
    device = torch.device("cuda")
    backend_kwargs.setdefault("output_srgb", False)
    backend = CustomCudaBackend(native_module=native_module.load_native_extension(), **backend_kwargs)
    service = ref.RendererService(backend, height=rig.height, width=rig.width, max_views=rig.viewmats.shape[0])
    service.initialize(stage=None, device=device)
    for sid, scene in scenes:
        service.load_scene(sid, **scene.to(device).as_kwargs())
    return service, backend


def _check_frame(out, want, cameras=None):
    """Bitwise equality with the oracle, on the listed cameras (all by default)."""
    pairs = (("rgb", want.rgb), ("depth", want.depth), ("alpha", want.alpha), ("semantic_id", want.semantic))
    for name, expected in pairs:
        got = out[name].cpu().numpy()
        if cameras is not None:
            got, expected = got[cameras], np.asarray(expected)[cameras]
        assert_bitwise_equal(got, expected, name)


def test_reference_service_renders_plain_config_with_capacity_growth():
    """10,000 Gaussians, one 256x256 camera (the plain single-camera
    workload): the reference backend starts with room for 512 visible
    records, overflows, grows its workspace and retries (cuda_backend.py:
    419-578), and the final frame equals the oracle bit for bit."""
    scene, rig = plain_workload()
    service, backend = _reference_camera_service(rig, [(0, scene)], visible_capacity_per_view=512,
                                                 intersections_per_visible=1.0, deterministic=True)
    device = torch.device("cuda")
    out = service.render(rig.viewmats.to(device), rig.intrinsics.to(device),
                         torch.zeros((1,), dtype=torch.int64, device=device))
    service.synchronize()
    want = render_oracle([(0, scene)], rig, [0])
    _check_frame(out, want)
    stats = backend.capacity_stats  # a property of the reference backend
    assert stats["last_render"]["status"] == "success"
    assert stats["last_render"]["retry_count"] >= 1
    counters = backend.read_counters()
    assert counters["visible_gaussians"] == want.visible
    assert counters["tile_intersections"] == want.intersections
    # The workspace contract the reference's diagnostics read: the sorted
    # record indices of every tile in values_out, tile ranges in tile_starts/
    # tile_ends.
    ws = service.workspace
    starts = ws["tile_starts"][:256].cpu().numpy()
    ends = ws["tile_ends"][:256].cpu().numpy()
    assert int((ends - starts).clip(min=0).sum()) == want.intersections
    service.shutdown()


def test_reference_service_multi_scene_active_subset_and_projection_cache():
    """Two scenes, five cameras of which three are active, through the
    reference service; the second identical render is a projection-cache
    hit (reuse_projection) and must give the same images."""
    a = synthetic_scene(6_000, seed=31, mean_half_extent=1.4, log_scale_mean=-3.4)
    b = synthetic_scene(9_000, seed=32, mean_half_extent=1.6, log_scale_mean=-3.6)
    rig = orbit_cameras(5, seed=9, radius=4.2, height_offset=0.4, width=80, height=56, focal=70.0)
    scene_ids = [7, 9, 9, 7, 9]
    active = [4, 0, 2]
    service, backend = _reference_camera_service(rig, [(7, a), (9, b)], enable_projection_cache=True)
    device = torch.device("cuda")
    view, intr = rig.viewmats.to(device), rig.intrinsics.to(device)
    ids = torch.tensor(scene_ids, dtype=torch.int64, device=device)
    active_t = torch.tensor(active, dtype=torch.int64, device=device)
    first = {k: v.clone() for k, v in service.render(view, intr, ids, active_camera_ids=active_t).items()}
    second = service.render(view, intr, ids, active_camera_ids=active_t)
    service.synchronize()
    want = render_oracle([(7, a), (9, b)], rig, scene_ids, active_ids=active)
    _check_frame(first, want, active)
    _check_frame(second, want, active)
    # The reference backend's inactive contract (cuda_backend.py:654-662).
    inactive = [c for c in range(5) if c not in active]
    assert torch.all(first["semantic_id"][inactive] == -1) and torch.all(first["alpha"][inactive] == 0)
    assert torch.all(torch.isinf(first["depth"][inactive]))
    service.shutdown()


def test_reference_service_chunked_logical_batch():
    """A six-camera logical batch submitted by the reference backend in
    physical chunks of two (cuda_backend.py:759-967)."""
    scene = synthetic_scene(7_000, seed=41, mean_half_extent=1.5, log_scale_mean=-3.5)
    rig = orbit_cameras(6, seed=4, radius=4.0, height_offset=0.6, width=64, height=48, focal=60.0)
    # The reference's chunked form runs with explicit capacity and a
    # fixed-capacity sort (cuda_backend.py:192-206).
    service, backend = _reference_camera_service(rig, [(3, scene)], max_physical_views=2, fixed_capacity_sort=True,
                                                 adaptive_capacity=False, max_visible_records=60_000,
                                                 max_intersections=400_000)
    device = torch.device("cuda")
    out = service.render(rig.viewmats.to(device), rig.intrinsics.to(device),
                         torch.full((6,), 3, dtype=torch.int64, device=device))
    service.synchronize()
    _check_frame(out, render_oracle([(3, scene)], rig, [3] * 6))
    service.shutdown()


def _f32(values, device):
    return torch.as_tensor(np.asarray(values), dtype=torch.float32).contiguous().to(device)


@pytest.mark.parametrize("name", lidar_cases.names())
def test_reference_lidar_service_matches_reference_oracle_golden(name):
    """The reference's GaussianLidarService + CudaLidarBackend on this
    library's LiDAR module, on the golden cases of the reference's LiDAR CPU
    oracle (experiments/lidar_cpu_oracle.py)."""
    ref, _, CudaLidarBackend = _reference_package()
    case = lidar_cases.load(name)
    device = torch.device("cuda")
    backend = CudaLidarBackend(native_module=load_lidar_extension())
    rays = _f32(case["rays"], device)
    sensors = _f32(case["sensors"], device)
    returns = case["kwargs"]["returns"]
    service = ref.GaussianLidarService(backend, max_sensors=sensors.shape[0], max_rays=rays.shape[0],
                                       returns=returns)
    service.initialize(stage=None, device=device)
    for sid, sc in case["scenes"].items():
        kwargs = {
            "means": _f32(sc["means"], device),
            "scales": _f32(sc["scales"], device),
            "rotations": _f32(sc["rotations"], device),
            "opacities": _f32(sc["opacities"], device),
            "semantic_ids": torch.as_tensor(sc["semantic_ids"], dtype=torch.int64).to(device),
        }
        for key in ("reflectivity", "surface_confidence"):
            if sc[key] is not None:
                kwargs[key] = _f32(sc[key], device)
        service.load_scene(sid, **kwargs)
    extra = {}
    if "scene_to_world" in case["kwargs"]:
        extra["scene_to_world"] = _f32(case["kwargs"]["scene_to_world"], device)
    if "active_sensor_ids" in case["kwargs"]:
        extra["active_sensor_ids"] = torch.as_tensor(case["kwargs"]["active_sensor_ids"],
                                                     dtype=torch.int64).to(device)
    out = service.render_lidar(rays, torch.as_tensor(case["times"], dtype=torch.int64).to(device), sensors,
                               torch.as_tensor(case["scene_ids"], dtype=torch.int64).to(device), **extra)
    service.synchronize()
    got = {k: v.cpu().numpy() for k, v in out.items()}
    want = case["expected"]
    for key in ("valid", "semantic_id", "return_count", "time_offset_ns"):
        np.testing.assert_array_equal(got[key], np.asarray(want[key]).astype(got[key].dtype), err_msg=key)
    valid = np.asarray(want["valid"]).astype(bool)
    np.testing.assert_allclose(got["range_m"][valid], want["range_m"][valid], rtol=0, atol=1e-4)
    np.testing.assert_allclose(got["intensity"][valid], want["intensity"][valid], rtol=0, atol=1e-4)
    assert np.all(np.isinf(got["range_m"][~valid]))
    service.shutdown()


def test_reference_lidar_service_revision_rebuilds_on_this_library():
    """Same-storage geometry edit + revise_scene through the reference
    service: the rebuilt acceleration sees the moved surfel."""
    ref, _, CudaLidarBackend = _reference_package()
    device = torch.device("cuda")
    backend = CudaLidarBackend(native_module=load_lidar_extension())
    service = ref.GaussianLidarService(backend, max_sensors=1, max_rays=1)
    service.initialize(stage=None, device=device)
    means = torch.tensor([[5.0, 0.0, 0.0]], device=device)
    scene = {
        "means": means,
        "scales": torch.tensor([[0.01, 0.5, 0.5]], device=device),
        "rotations": torch.tensor([[1.0, 0.0, 0.0, 0.0]], device=device),
        "opacities": torch.tensor([0.99], device=device),
        "semantic_ids": torch.tensor([4], dtype=torch.int64, device=device),
    }
    service.load_scene(1, **scene)
    args = (torch.tensor([[1.0, 0.0, 0.0]], device=device), torch.zeros((1,), dtype=torch.int64, device=device),
            torch.eye(4, device=device)[None].contiguous(), torch.ones((1,), dtype=torch.int64, device=device))
    before = float(service.render_lidar(*args)["range_m"][0, 0, 0])
    means[0, 0] = 8.0
    service.revise_scene(1, revision=1)
    after = float(service.render_lidar(*args)["range_m"][0, 0, 0])
    assert math.isclose(before, 5.0, abs_tol=0.02) and math.isclose(after, 8.0, abs_tol=0.02)
    service.shutdown()
