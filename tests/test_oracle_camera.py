"""Known-answer tests of the CPU camera oracle (no GPU needed).

These pin the restatement to hand-derived values of the reference equation
(renderer_cuda.cu:179-201,287-490,1973-2305) and to the known answers the
reference's own CUDA smoke checks (scripts/deterministic_cuda_smoke.py:33-180:
equal-depth order = Gaussian id, centre semantic = lowest id).
"""

from __future__ import annotations

import math

import numpy as np
import pytest

from oracle import camera as oc
from vgr_b200.workloads import CameraRig, pinhole, plain_workload


def test_exp_log_srgb_accuracy():
    for x in np.linspace(-20.0, 0.0, 2001, dtype=np.float32):
        got, want = oc.exp(float(x)), math.exp(float(x))
        assert abs(got - want) <= 4e-7 * want
    for y in np.geomspace(1.0, 300.0, 2001).astype(np.float32):
        got, want = oc.log(float(y)), math.log(float(y))
        assert abs(got - want) <= 4e-7 * max(1.0, abs(want))
    for v in np.linspace(0.0, 1.0, 501, dtype=np.float32):
        v = float(v)
        want = 12.92 * v if v <= 0.0031308 else 1.055 * v ** (1 / 2.4) - 0.055
        assert abs(oc.srgb(v) - want) <= 2e-6


def test_covariance_of_axis_aligned_gaussian():
    cov = oc.precompute_covariances([[0.1, 0.2, 0.3]], [[2.0, 0.0, 0.0, 0.0]])
    np.testing.assert_allclose(cov[0], [0.01, 0.0, 0.0, 0.04, 0.0, 0.09], rtol=1e-6, atol=1e-9)


def _single(opacity=0.8, scale=0.05, depth=2.0, w=32, h=32, f=32.0, eps=0.3, ray=False, centre=None):
    view = np.eye(4, dtype=np.float32)[None]
    cx, cy = (w / 2, h / 2) if centre is None else centre
    k = pinhole(1, f, f, cx, cy).numpy()
    rot = np.array([[1.0, 0.0, 0.0, 0.0]], dtype=np.float32)
    cov = oc.precompute_covariances([[scale, scale, scale]], rot)
    return oc.render(
        means=[[0.0, 0.0, depth]],
        covariances=cov,
        opacities=[opacity],
        features=[[0.2, 0.4, 0.6]],
        semantic_ids=[7],
        registered_scene_ids=[0],
        scene_offsets=[0, 1],
        viewmats=view,
        intrinsics=k,
        camera_scene_ids=[0],
        height=h,
        width=w,
        covariance_epsilon=eps,
        with_tiles=True,
        ray_gaussian_evaluation=ray,
    )


def test_single_gaussian_analytic_alpha():
    opacity, scale, depth, f = 0.8, 0.05, 2.0, 32.0
    res = _single(opacity, scale, depth, f=f)
    # Screen covariance: (f s / z)^2 + eps on both axes, no cross term.
    var = (f * scale / depth) ** 2 + 0.3
    for px, py in [(16, 16), (17, 16), (18, 18), (15, 14)]:
        dx, dy = px + 0.5 - 16.0, py + 0.5 - 16.0
        alpha = min(0.99, opacity * math.exp(-0.5 * (dx * dx + dy * dy) / var))
        expected_alpha = alpha if alpha >= 1 / 255 else 0.0
        assert res.alpha[0, py, px, 0] == pytest.approx(expected_alpha, rel=2e-6, abs=1e-7)
        if expected_alpha > 0:
            np.testing.assert_allclose(res.rgb[0, py, px], np.array([0.2, 0.4, 0.6]) * alpha, rtol=3e-6)
            assert res.depth[0, py, px, 0] == pytest.approx(depth, rel=1e-6)
            assert res.semantic[0, py, px, 0] == (7 if alpha >= 0.01 else -1)
    assert res.visible == 1
    # Radius ceil(min(3.33, sqrt(2 ln(255 o))) sqrt(var)) covers one 16-px tile
    # around the centre at (16,16) -> tiles (0..1) x (0..1).
    ext = min(3.33, math.sqrt(2.0 * math.log(opacity * 255.0)))
    radius = math.ceil(ext * math.sqrt(var))
    lo = max(0, math.floor((16.0 - radius) / 16))
    hi = min(2, math.ceil((16.0 + radius) / 16))
    assert res.intersections == (hi - lo) ** 2
    assert res.tile_counts.sum() == res.intersections


def test_exact_ray_single_gaussian_analytic_alpha():
    # Exact-ray mode (renderer_cuda.cu:203-245): for an isotropic Gaussian of
    # std s at (0, 0, z) and the pixel ray d = (nx, ny, 1), the squared
    # Mahalanobis distance from the mean to the ray is
    # z^2 (nx^2 + ny^2) / ((1 + nx^2 + ny^2) s^2); no screen-space dilation,
    # no 1/255 cut, no 0.99 clamp.  m^T P m - (d^T P m)^2 / d^T P d cancels
    # in float (the reference's evaluation), so alpha holds to ~1e-4.
    opacity, scale, depth, f, sigma = 0.3, 0.05, 2.0, 32.0, 3.33
    res = _single(opacity, scale, depth, f=f, ray=True)
    below_cut = 0
    for px, py in [(16, 16), (17, 16), (18, 18), (15, 14), (18, 16), (19, 16), (13, 17)]:
        nx, ny = (px + 0.5 - 16.0) / f, (py + 0.5 - 16.0) / f
        m2 = depth * depth * (nx * nx + ny * ny) / ((1 + nx * nx + ny * ny) * scale * scale)
        alpha = min(1.0, opacity * math.exp(-0.5 * m2)) if m2 <= sigma * sigma else 0.0
        below_cut += 0 < alpha < 1 / 255
        assert res.alpha[0, py, px, 0] == pytest.approx(alpha, rel=5e-4, abs=1e-9), (px, py)
        if alpha > 0:
            np.testing.assert_allclose(res.rgb[0, py, px], np.array([0.2, 0.4, 0.6]) * alpha, rtol=5e-4)
            assert res.depth[0, py, px, 0] == pytest.approx(depth, rel=1e-5)
    assert below_cut >= 1  # the screen-space 1/255 cut does not apply
    assert res.visible == 1


def test_exact_ray_opaque_gaussian_terminates_after_blending():
    # alpha = min(1, o exp(-m^2/2)) is 1 up to float cancellation on the ray
    # through the mean (pixel (16, 16) with the principal point at its
    # centre): the pixel blends the record and stops (T <= 1e-4), where the
    # screen-space path clamps alpha at 0.99.
    res = _single(opacity=1.0, scale=0.2, depth=2.0, ray=True, centre=(16.5, 16.5))
    assert res.alpha[0, 16, 16, 0] > 1.0 - 1e-4
    np.testing.assert_allclose(res.rgb[0, 16, 16], [0.2, 0.4, 0.6], rtol=1e-4)
    screen = _single(opacity=1.0, scale=0.2, depth=2.0, centre=(16.5, 16.5))
    assert screen.alpha[0, 16, 16, 0] == pytest.approx(0.99, rel=1e-6)


def test_gaussian_behind_camera_and_low_opacity_are_culled():
    res = _single(depth=-1.0)
    assert res.visible == 0 and res.intersections == 0
    assert np.all(res.alpha == 0) and np.all(np.isinf(res.depth)) and np.all(res.semantic == -1)
    res = _single(opacity=1.0 / 256.0)
    assert res.visible == 0


def test_equal_depth_ties_order_by_gaussian_id():
    count = 64
    means = np.zeros((count, 3), np.float32)
    means[:, 2] = 5.0
    cov = oc.precompute_covariances(np.full((count, 3), 0.03, np.float32), np.tile([[1.0, 0, 0, 0]], (count, 1)))
    view = np.eye(4, dtype=np.float32)[None].copy()
    view[0, 2, 3] = -4.0
    res = oc.render(
        means=means,
        covariances=cov,
        opacities=np.full((count,), 0.2, np.float32),
        features=np.tile([[1.0, 0.0, 0.0]], (count, 1)),
        semantic_ids=np.arange(1000, 1000 + count),
        registered_scene_ids=[73],
        scene_offsets=[0, count],
        viewmats=view,
        intrinsics=pinhole(1, 64.0, 64.0, 32.0, 32.0).numpy(),
        camera_scene_ids=[73],
        height=64,
        width=64,
        support_sigma=3.0,
        with_tiles=True,
    )
    starts = np.concatenate([[0], np.cumsum(res.tile_counts)])
    centre = 2 * 4 + 2
    ids = res.sorted_gaussian_ids[starts[centre] : starts[centre + 1]]
    np.testing.assert_array_equal(ids, np.arange(count))
    assert res.semantic[0, 32, 32, 0] == 1000


def test_plain_workload_is_deterministic_and_finite():
    scene, rig = plain_workload()
    cov = oc.precompute_covariances(scene.scales.numpy(), scene.rotations.numpy())
    kwargs = dict(
        means=scene.means.numpy(),
        covariances=cov,
        opacities=scene.opacities.numpy(),
        features=scene.features.numpy(),
        semantic_ids=scene.semantic_ids.numpy(),
        registered_scene_ids=[0],
        scene_offsets=[0, scene.means.shape[0]],
        viewmats=rig.viewmats.numpy(),
        intrinsics=rig.intrinsics.numpy(),
        camera_scene_ids=[0],
        height=rig.height,
        width=rig.width,
    )
    a = oc.render(**kwargs, threads=1)
    b = oc.render(**kwargs, threads=4)
    for x, y in ((a.rgb, b.rgb), (a.alpha, b.alpha), (a.depth, b.depth), (a.semantic, b.semantic)):
        np.testing.assert_array_equal(x, y)
    assert np.isfinite(a.rgb).all() and (a.alpha >= 0).all() and (a.alpha <= 1).all()
    assert a.visible > 1000 and a.intersections >= a.visible
