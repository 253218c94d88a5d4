"""The allocation-free entry point renders exactly what vgr_render renders.

vgr_render_static_scratch exists for callers that cannot allocate device
memory while they render (a plug-in whose host owns every allocation, a
real-time loop, code being captured into a CUDA graph): it takes the same
inputs, outputs and workspace buffers as vgr_render but keeps its scratch in
a fixed array inside the library.  These tests call both entry points
through the C ABI on the same inputs and require bit-identical outputs and
counters, twice in a row (the shared array keeps the previous call's
contents, so the second call checks that everything is cleared), that a
render of exactly vgr_static_scratch_max_cameras() cameras runs while one more
camera is refused with a clear error before anything is launched, and that
reuse_projection (which would read another call's plans from the shared
array) is refused.  The file name sorts last so a run that stops at the first failure has
already run every other test.
"""

from __future__ import annotations

import ctypes

import pytest
import torch

from vgr_b200 import CustomCudaBackend, RendererService, _native
from vgr_b200.workloads import CameraRig, orbit_cameras, pinhole, synthetic_scene

pytestmark = pytest.mark.gpu


def _setup():
    device = torch.device("cuda")
    scene = synthetic_scene(30_000, seed=17, mean_half_extent=1.5, log_scale_mean=-3.4, sh_degree=1)
    rig = orbit_cameras(3, seed=5, radius=4.0, height_offset=0.7, width=96, height=72, focal=80.0)
    backend = CustomCudaBackend(output_srgb=True, sh_degree=1)
    service = RendererService(backend, height=rig.height, width=rig.width, max_views=3)
    service.initialize(stage=None, device=device)
    service.load_scene(4, **scene.to(device).as_kwargs())
    # Size the workspace with one ordinary render.
    service.render(rig.viewmats.to(device), rig.intrinsics.to(device), torch.tensor([4, 4, 4], device=device))
    service.synchronize()
    return device, rig, backend


def _structs(device, rig, backend, intersection_capacity=None, max_scene_gaussians=None, tiles=None):
    packed = backend._packed_scene
    ws = backend.workspace
    batch = rig.viewmats.shape[0]
    viewmats = rig.viewmats.to(device)
    intrinsics = rig.intrinsics.to(device)
    env = torch.eye(4, device=device).repeat(batch, 1, 1).contiguous()
    scene_ids = torch.full((batch,), 4, dtype=torch.int64, device=device)
    icap = intersection_capacity or backend.current_intersection_capacity
    vcap = backend.current_visible_capacity
    tiles = max(tiles or 0, ws["tile_starts"].numel())
    buffers = {
        "records": torch.empty((vcap, 12), dtype=torch.float32, device=device),
        "keys_in": torch.empty((icap,), dtype=torch.uint64, device=device),
        "keys_out": torch.empty((icap,), dtype=torch.uint64, device=device),
        "values_in": torch.empty((icap,), dtype=torch.int32, device=device),
        "values_out": torch.empty((icap,), dtype=torch.int32, device=device),
        "tile_starts": torch.empty((tiles,), dtype=torch.int32, device=device),
        "tile_ends": torch.empty((tiles,), dtype=torch.int32, device=device),
        "counters": torch.empty((5,), dtype=torch.int64, device=device),
        "rgb": torch.empty((batch, rig.height, rig.width, 3), device=device),
        "depth": torch.empty((batch, rig.height, rig.width, 1), device=device),
        "alpha": torch.empty((batch, rig.height, rig.width, 1), device=device),
        "semantic": torch.empty((batch, rig.height, rig.width, 1), dtype=torch.int64, device=device),
        "_keep": [viewmats, intrinsics, env, scene_ids],
    }
    scene = _native.VgrScene(
        means=packed["means"].data_ptr(),
        covariances=packed["covariances"].data_ptr(),
        opacities=packed["opacities"].data_ptr(),
        features=packed["features"].data_ptr(),
        feature_width=packed["features"].shape[1],
        semantic_ids=packed["semantic_ids"].data_ptr(),
        registered_scene_ids=packed["registered_scene_ids"].data_ptr(),
        scene_offsets=packed["scene_offsets"].data_ptr(),
        scene_count=1,
        gaussian_count=packed["means"].shape[0],
        max_scene_gaussians=max_scene_gaussians or packed["means"].shape[0],
    )
    cams = _native.VgrCameras(
        viewmats=viewmats.data_ptr(),
        intrinsics=intrinsics.data_ptr(),
        env_xforms=env.data_ptr(),
        camera_scene_ids=scene_ids.data_ptr(),
        active_camera_ids=None,
        batch=batch,
        active_count=batch,
    )
    outs = _native.VgrOutputs(
        rgb=buffers["rgb"].data_ptr(),
        depth=buffers["depth"].data_ptr(),
        alpha=buffers["alpha"].data_ptr(),
        semantic=buffers["semantic"].data_ptr(),
    )
    workspace = _native.VgrWorkspace(
        records=buffers["records"].data_ptr(),
        visible_capacity=vcap,
        keys_in=buffers["keys_in"].data_ptr(),
        keys_out=buffers["keys_out"].data_ptr(),
        values_in=buffers["values_in"].data_ptr(),
        values_out=buffers["values_out"].data_ptr(),
        intersection_capacity=icap,
        tile_starts=buffers["tile_starts"].data_ptr(),
        tile_ends=buffers["tile_ends"].data_ptr(),
        tile_capacity=tiles,
        counters=buffers["counters"].data_ptr(),
        scratch=ws["scratch"].data_ptr(),
        scratch_bytes=ws["scratch"].numel(),
    )
    options = _native.VgrRenderOptions(
        height=rig.height,
        width=rig.width,
        near_plane=0.01,
        far_plane=100.0,
        gaussian_support_sigma=3.33,
        covariance_epsilon=0.3,
        semantic_min_alpha=0.01,
        tile_size=16,
        output_srgb=1,
        full_sensor_output=1,
        sh_degree=1,
        sorted_buffer_hint=1,
    )
    return scene, cams, outs, workspace, options, buffers


def _call(entry, device, structs):
    scene, cams, outs, workspace, options, _ = structs
    selector = ctypes.c_int64(-1)
    stream = torch.cuda.current_stream(device).cuda_stream
    code = entry(scene, cams, outs, workspace, options, stream, selector)
    return code, selector.value


def test_static_scratch_matches_vgr_render_twice_in_a_row():
    device, rig, backend = _setup()
    lib = _native.load_library()
    reference = _structs(device, rig, backend)
    code, selector = _call(lib.vgr_render, device, reference)
    assert code == 0, _native.last_error()
    torch.cuda.synchronize()
    expected = {k: reference[5][k].clone() for k in ("rgb", "depth", "alpha", "semantic", "counters")}
    assert int(expected["counters"][1]) > 0

    candidate = _structs(device, rig, backend)
    for _ in range(2):
        for name in ("rgb", "depth", "alpha"):
            candidate[5][name].fill_(float("nan"))
        candidate[5]["semantic"].fill_(-7)
        candidate[5]["counters"].fill_(-1)
        code, static_selector = _call(lib.vgr_render_static_scratch, device, candidate)
        assert code == 0, _native.last_error()
        torch.cuda.synchronize()
        assert static_selector == selector
        for name, want in expected.items():
            got = candidate[5][name]
            if got.is_floating_point():
                assert torch.equal(got.view(torch.int32), want.view(torch.int32)), name
            else:
                assert torch.equal(got, want), name


def _far_side_rig(count):
    """``count`` one-pixel cameras whose scene lies behind them (nothing
    visible): the render's cost is the per-camera setup, which is what the
    static array's size limits."""
    view = torch.eye(4).repeat(count, 1, 1)
    view[:, 2, 3] = -5.0
    return CameraRig(view.contiguous(), pinhole(count, 1.0, 1.0, 0.5, 0.5), 1, 1)


def test_static_scratch_renders_at_its_camera_limit_and_refuses_one_more():
    device, _, backend = _setup()
    lib = _native.load_library()
    limit = lib.vgr_static_scratch_max_cameras()
    assert 95_000 < limit < 96_000
    structs = _structs(device, _far_side_rig(limit), backend, tiles=limit)
    structs[5]["alpha"].fill_(float("nan"))
    code, _ = _call(lib.vgr_render_static_scratch, device, structs)
    assert code == 0, _native.last_error()
    torch.cuda.synchronize()
    assert int(structs[5]["counters"][0]) == 0 and int(structs[5]["counters"][1]) == 0
    assert torch.all(structs[5]["alpha"] == 0.0)

    over = _structs(device, _far_side_rig(limit + 1), backend, tiles=limit + 1)
    over[5]["counters"].fill_(-1)
    code, _ = _call(lib.vgr_render_static_scratch, device, over)
    assert code == _native.VGR_ERR_SCRATCH_TOO_SMALL
    assert "static array" in _native.last_error()
    torch.cuda.synchronize()
    assert torch.all(over[5]["counters"] == -1)  # nothing was launched


def test_static_scratch_refuses_reuse_projection():
    device, rig, backend = _setup()
    lib = _native.load_library()
    structs = _structs(device, rig, backend)
    structs[4].reuse_projection = 1
    structs[5]["counters"].fill_(-1)
    code, _ = _call(lib.vgr_render_static_scratch, device, structs)
    assert code == _native.VGR_ERR_INVALID_ARGUMENT
    assert "reuse_projection" in _native.last_error()
    torch.cuda.synchronize()
    assert torch.all(structs[5]["counters"] == -1)
