"""Differentiable camera form: gradients of the hand-written CUDA backward
against float64 automatic differentiation of the same equation, which is in
turn checked against float64 central finite differences.

The reference has no backward (its gradients come from gsplat, which is not
available here), so parity for gradients is pinned by the float64 statement
in diff_reference.py: the FD check (CPU) shows that its autograd gradients
are the derivatives of the forward; the GPU tests show that the CUDA forward
matches it within 1e-4 and that the CUDA gradients match its gradients to a
relative L2 error below 2e-3 per parameter tensor.
"""

from __future__ import annotations

import pytest
import torch

from diff_reference import render_reference, weighted_loss
from vgr_b200.workloads import look_at_viewmats, pinhole

SIZE = 32
NAMES = ("means", "log_scales", "rotations", "opacity_logits", "features")


def _scene(seed: int, count: int = 64, sh_degree: int = 3) -> dict[str, torch.Tensor]:
    gen = torch.Generator().manual_seed(seed)
    k = 1 if sh_degree < 0 else (sh_degree + 1) ** 2
    features = torch.randn((count, k * 3), generator=gen) * 0.25
    features[:, :3] = torch.rand((count, 3), generator=gen) * (1.2 if sh_degree < 0 else 2.4) - (
        0.0 if sh_degree < 0 else 0.9
    )
    return {
        "means": (torch.rand((count, 3), generator=gen) - 0.5) * 1.2,
        "log_scales": torch.randn((count, 3), generator=gen) * 0.3 - 2.2,
        "rotations": torch.randn((count, 4), generator=gen),
        "opacity_logits": torch.randn((count,), generator=gen) * 1.2,
        "features": features,
    }


def _cameras(count: int = 2, seed: int = 3) -> tuple[torch.Tensor, torch.Tensor]:
    gen = torch.Generator().manual_seed(seed)
    angle = torch.rand((count,), generator=gen, dtype=torch.float64) * 6.283
    eyes = torch.stack((3.0 * torch.cos(angle), 0.4 + 0.3 * torch.rand((count,), generator=gen, dtype=torch.float64),
                        3.0 * torch.sin(angle)), dim=1)
    view = look_at_viewmats(eyes, torch.zeros((count, 3), dtype=torch.float64))
    return view, pinhole(count, 38.0, 38.0, SIZE / 2.0, SIZE / 2.0)


def _weights(count: int, seed: int = 11) -> tuple[torch.Tensor, torch.Tensor, torch.Tensor]:
    gen = torch.Generator().manual_seed(seed)
    return (
        torch.randn((count, SIZE, SIZE, 3), generator=gen, dtype=torch.float64),
        torch.randn((count, SIZE, SIZE, 1), generator=gen, dtype=torch.float64) * 0.1,
        torch.randn((count, SIZE, SIZE, 1), generator=gen, dtype=torch.float64),
    )


def _reference_grads(scene, view, intr, weights, sh_degree):
    params = {k: v.double().clone().requires_grad_(True) for k, v in scene.items()}
    rgb, depth, alpha = render_reference(
        *(params[k] for k in NAMES), view.double(), intr.double(), SIZE, SIZE, sh_degree=sh_degree
    )
    loss = weighted_loss(rgb, depth, alpha, weights)
    loss.backward()
    return (rgb.detach(), depth.detach(), alpha.detach()), {k: params[k].grad for k in NAMES}


def test_reference_gradients_match_central_differences():
    # CPU: the float64 statement's autograd gradients are the derivatives of
    # its forward (central differences, h = 1e-6, on a sample of entries).
    sh_degree = 3
    scene = _scene(21, count=24, sh_degree=sh_degree)
    view, intr = _cameras(1)
    weights = tuple(w[:1] for w in _weights(1))
    _, grads = _reference_grads(scene, view, intr, weights, sh_degree)
    base = {k: v.double() for k, v in scene.items()}

    def loss_at(params):
        out = render_reference(*(params[k] for k in NAMES), view.double(), intr.double(), SIZE, SIZE,
                               sh_degree=sh_degree)
        return float(weighted_loss(*out, weights))

    gen = torch.Generator().manual_seed(5)
    h = 1e-6
    checked = 0
    for name in NAMES:
        flat = base[name].reshape(-1)
        picks = torch.randperm(flat.numel(), generator=gen)[:6]
        for idx in picks.tolist():
            plus = {k: v.clone() for k, v in base.items()}
            minus = {k: v.clone() for k, v in base.items()}
            plus[name].view(-1)[idx] += h
            minus[name].view(-1)[idx] -= h
            fd = (loss_at(plus) - loss_at(minus)) / (2 * h)
            an = float(grads[name].reshape(-1)[idx])
            assert abs(fd - an) <= 1e-6 + 1e-5 * max(abs(fd), abs(an)), (name, idx, fd, an)
            checked += 1
    assert checked == 6 * len(NAMES)


def test_reference_forward_matches_the_oracle():
    # CPU: the float64 statement renders what the bit-exact C oracle (the
    # camera equation the CUDA forward reproduces bit for bit) renders.
    from helpers import render_oracle
    from vgr_b200.workloads import CameraRig, SceneTensors

    sh_degree = 3
    scene = _scene(31, sh_degree=sh_degree)
    view, intr = _cameras(2, seed=9)
    rgb, depth, alpha = render_reference(
        *(scene[k].double() for k in NAMES), view.double(), intr.double(), SIZE, SIZE, sh_degree=sh_degree
    )
    activated = SceneTensors(
        means=scene["means"],
        scales=torch.exp(scene["log_scales"]),
        rotations=scene["rotations"],
        opacities=torch.sigmoid(scene["opacity_logits"]),
        features=scene["features"],
        semantic_ids=torch.zeros(scene["means"].shape[0], dtype=torch.int64),
    )
    cpu = render_oracle([(0, activated)], CameraRig(view, intr, SIZE, SIZE), [0, 0], sh_degree=sh_degree)
    assert float(torch.max(torch.abs(rgb - torch.from_numpy(cpu.rgb).double()))) < 1e-4
    assert float(torch.max(torch.abs(alpha - torch.from_numpy(cpu.alpha).double()))) < 1e-4
    finite = torch.isfinite(depth)
    oracle_depth = torch.from_numpy(cpu.depth).double()
    assert torch.equal(torch.isfinite(oracle_depth), finite)
    assert float(torch.max(torch.abs(depth[finite] - oracle_depth[finite]))) < 1e-3
    assert float(alpha.max()) > 0.5  # the scene covers pixels


def _gpu_case(sh_degree: int, tile_size: int, seed: int):
    from vgr_b200.differentiable import DifferentiableRenderer

    scene = _scene(seed, sh_degree=sh_degree)
    view, intr = _cameras(2, seed=seed + 1)
    weights = _weights(2, seed=seed + 2)
    ref_out, ref_grads = _reference_grads(scene, view, intr, weights, sh_degree)
    renderer = DifferentiableRenderer(height=SIZE, width=SIZE, sh_degree=sh_degree, tile_size=tile_size)
    params = {k: v.cuda().requires_grad_(True) for k, v in scene.items()}
    rgb, depth, alpha = renderer.render(*(params[k] for k in NAMES), view.cuda(), intr.cuda())
    loss = weighted_loss(rgb, depth, alpha, tuple(w.float().cuda() for w in weights))
    loss.backward()
    return (rgb, depth, alpha), ref_out, {k: params[k].grad for k in NAMES}, ref_grads


@pytest.mark.gpu
@pytest.mark.parametrize("sh_degree,tile_size", [(3, 16), (3, 8), (0, 16), (-1, 16)])
def test_gpu_gradients_match_float64_autograd(sh_degree, tile_size):
    (rgb, depth, alpha), (r_rgb, r_depth, r_alpha), grads, ref = _gpu_case(sh_degree, tile_size, 40 + sh_degree)
    # Forward: the training forward matches the float64 statement.
    assert torch.max(torch.abs(rgb.double().cpu() - r_rgb)) < 1e-4
    assert torch.max(torch.abs(alpha.double().cpu() - r_alpha)) < 1e-4
    finite = torch.isfinite(r_depth)
    assert torch.equal(torch.isfinite(depth.cpu()), finite)
    assert torch.max(torch.abs(depth.double().cpu()[finite] - r_depth[finite])) < 1e-4 * 10
    for name in NAMES:
        got = grads[name].double().cpu()
        want = ref[name]
        scale = float(torch.linalg.norm(want))
        assert scale > 0, name
        err = float(torch.linalg.norm(got - want)) / scale
        assert err < 2e-3, (name, err)


@pytest.mark.gpu
def test_gpu_backward_needs_the_last_frame():
    from vgr_b200.differentiable import DifferentiableRenderer

    scene = _scene(7)
    view, intr = _cameras(1)
    renderer = DifferentiableRenderer(height=SIZE, width=SIZE, sh_degree=3)
    params = {k: v.cuda().requires_grad_(True) for k, v in scene.items()}
    first = renderer.render(*(params[k] for k in NAMES), view.cuda(), intr.cuda())
    second = renderer.render(*(params[k] for k in NAMES), view.cuda(), intr.cuda())
    with pytest.raises(RuntimeError, match="one frame in flight"):
        first[0].sum().backward()
    second[0].sum().backward()
    assert params["means"].grad is not None and torch.isfinite(params["means"].grad).all()


@pytest.mark.gpu
def test_gpu_photometric_loss_matches_torch():
    from vgr_b200.differentiable import photometric_loss

    gen = torch.Generator().manual_seed(2)
    rgb = torch.rand((2, 8, 8, 3), generator=gen).cuda().requires_grad_(True)
    depth = (torch.rand((2, 8, 8, 1), generator=gen) * 5).cuda()
    depth[0, 0, 0, 0] = float("inf")
    depth = depth.requires_grad_(True)
    t_rgb = torch.rand((2, 8, 8, 3), generator=gen).cuda()
    t_depth = (torch.rand((2, 8, 8, 1), generator=gen) * 5).cuda()
    t_depth[1, 2, 3, 0] = float("inf")
    loss = photometric_loss(rgb, depth, t_rgb, t_depth, 0.1)
    loss.backward()
    r = rgb.detach().clone().requires_grad_(True)
    d = depth.detach().clone().requires_grad_(True)
    finite = torch.isfinite(d) & torch.isfinite(t_depth)
    diff = torch.where(finite, d - torch.where(finite, t_depth, torch.zeros_like(t_depth)), torch.zeros_like(d))
    want = ((r - t_rgb) ** 2).mean() + 0.1 * diff.abs().mean()
    want.backward()
    assert abs(float(loss.detach()) - float(want.detach())) < 1e-6
    assert torch.allclose(rgb.grad, r.grad, rtol=1e-5, atol=1e-8)
    assert torch.allclose(depth.grad, d.grad, rtol=1e-5, atol=1e-8)


@pytest.mark.gpu
def test_gpu_deferred_capacity_check_raises_and_regrows():
    from vgr_b200.differentiable import DifferentiableRenderer

    scene = _scene(8)
    view, intr = _cameras(2)
    sync = DifferentiableRenderer(height=SIZE, width=SIZE, sh_degree=3, tile_size=4)
    deferred = DifferentiableRenderer(height=SIZE, width=SIZE, sh_degree=3, tile_size=4, capacity_check="deferred")
    grads = []
    for renderer in (sync, deferred):
        params = {k: v.cuda().requires_grad_(True) for k, v in scene.items()}
        for _ in range(2):  # the first frame calibrates, the second is checked late
            rgb, depth, alpha = renderer.render(*(params[k] for k in NAMES), view.cuda(), intr.cuda())
            (rgb.sum() + alpha.sum()).backward()
        grads.append(params["means"].grad.clone())
    assert torch.allclose(grads[0], grads[1], rtol=1e-5, atol=1e-6)
    # Much larger Gaussians overflow the calibrated intersection capacity.
    big = dict(scene)
    big["log_scales"] = scene["log_scales"] + 2.5
    params = {k: v.cuda().requires_grad_(True) for k, v in big.items()}
    rgb, depth, alpha = deferred.render(*(params[k] for k in NAMES), view.cuda(), intr.cuda())
    with pytest.raises(RuntimeError, match="overflowed"):
        rgb.sum().backward()
    rgb, depth, alpha = deferred.render(*(params[k] for k in NAMES), view.cuda(), intr.cuda())
    rgb.sum().backward()
    assert torch.isfinite(params["means"].grad).all()


@pytest.mark.gpu
@pytest.mark.parametrize("capacity_check", ["sync", "deferred"])
def test_gpu_list_budget_recomputes_chunks_with_the_same_gradients(capacity_check):
    # A budget far below one camera's lists: the forward renders one camera
    # at a time and the backward recomputes each camera's sorted lists.
    from vgr_b200.differentiable import DifferentiableRenderer

    scene = _scene(77, count=400, sh_degree=3)
    view, intr = _cameras(5, seed=78)
    weights = tuple(w.float().cuda() for w in _weights(5, seed=79))
    results = []
    for budget in (None, 1):
        renderer = DifferentiableRenderer(height=SIZE, width=SIZE, sh_degree=3, tile_size=8,
                                          list_budget_bytes=budget, capacity_check=capacity_check)
        params = {k: v.cuda().requires_grad_(True) for k, v in scene.items()}
        for _ in range(3):  # later frames use the learned per-camera size (and deferred checks)
            for p in params.values():
                p.grad = None
            out = renderer.render(*(params[k] for k in NAMES), view.cuda(), intr.cuda())
            weighted_loss(*out, weights).backward()
        results.append(([t.detach().clone() for t in out], {k: params[k].grad.clone() for k in NAMES},
                        renderer._pending["chunks"]))
    (out_a, grads_a, chunks_a), (out_b, grads_b, chunks_b) = results
    assert chunks_a == [(0, 5)] and len(chunks_b) == 5
    for a, b in zip(out_a, out_b):
        assert torch.equal(a, b)  # the forward is the same render, camera by camera
    for name in NAMES:
        # Per-camera partial sums added in another order: float rounding only.
        torch.testing.assert_close(grads_b[name], grads_a[name], rtol=1e-4, atol=1e-6)
