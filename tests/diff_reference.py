"""Float64 PyTorch statement of the differentiable camera form (test helper).

A dense restatement of the image formation the native training forward
computes -- activations (exp scales, normalised WXYZ quaternion, sigmoid
opacity), the EWA projection of renderer_cuda.cu:287-490 (clamped Jacobian
point, covariance epsilon, opacity/near/far/determinant/radius/off-screen
culls), real SH colour through degree 3 with the +0.5 offset and the clamp
at zero, and the front-to-back compositor of renderer_cuda.cu:1973-2305
(alpha = min(0.99, o exp(power)), -20 <= power <= 0, alpha >= 1/255, stop
before a record whose next transmittance is <= 1e-4, depth = sum(w z) / alpha
or +inf) -- evaluated for every (pixel, Gaussian) pair in float64 so that
torch.autograd gives the exact gradients the hand-written CUDA backward is
compared with.  Order is (depth, Gaussian id).  Discrete decisions (culls,
thresholds) are taken on the float64 values and carry no gradient.
"""

from __future__ import annotations

import math

import torch

ALPHA_THRESHOLD = 1.0 / 255.0
MAX_ALPHA = 0.99
TRANSMITTANCE_THRESHOLD = 1.0e-4

SH_C0 = 0.28209479177387814
SH_C1 = 0.4886025119029199
SH_C2 = (1.0925484305920792, -1.0925484305920792, 0.31539156525252005, -1.0925484305920792, 0.5462742152960396)
SH_C3 = (
    -0.5900435899266435,
    2.890611442640554,
    -0.4570457994644658,
    0.3731763325901154,
    -0.4570457994644658,
    1.445305721320277,
    -0.5900435899266435,
)


def quaternion_rotation(q: torch.Tensor) -> torch.Tensor:
    """Rotation matrices [G,3,3] of WXYZ quaternions [G,4] of any norm."""
    n = q / torch.sqrt(torch.clamp((q * q).sum(-1, keepdim=True), min=1e-20))
    w, x, y, z = n.unbind(-1)
    rows = [
        1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y),
        2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x),
        2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y),
    ]
    return torch.stack(rows, -1).reshape(q.shape[0], 3, 3)


def sh_basis(dirs: torch.Tensor, degree: int) -> torch.Tensor:
    x, y, z = dirs.unbind(-1)
    basis = [torch.full_like(x, SH_C0)]
    if degree >= 1:
        basis += [-SH_C1 * y, SH_C1 * z, -SH_C1 * x]
    if degree >= 2:
        xx, yy, zz = x * x, y * y, z * z
        basis += [
            SH_C2[0] * x * y,
            SH_C2[1] * y * z,
            SH_C2[2] * (2 * zz - xx - yy),
            SH_C2[3] * x * z,
            SH_C2[4] * (xx - yy),
        ]
    if degree >= 3:
        basis += [
            SH_C3[0] * y * (3 * xx - yy),
            SH_C3[1] * x * y * z,
            SH_C3[2] * y * (4 * zz - xx - yy),
            SH_C3[3] * z * (2 * zz - 3 * xx - 3 * yy),
            SH_C3[4] * x * (4 * zz - xx - yy),
            SH_C3[5] * z * (xx - yy),
            SH_C3[6] * x * (xx - 3 * yy),
        ]
    return torch.stack(basis, -1)


def render_reference(
    means: torch.Tensor,
    log_scales: torch.Tensor,
    rotations: torch.Tensor,
    opacity_logits: torch.Tensor,
    features: torch.Tensor,
    viewmats: torch.Tensor,
    intrinsics: torch.Tensor,
    height: int,
    width: int,
    *,
    sh_degree: int = 3,
    near_plane: float = 0.01,
    far_plane: float = 100.0,
    support_sigma: float = 3.33,
    covariance_epsilon: float = 0.3,
) -> tuple[torch.Tensor, torch.Tensor, torch.Tensor]:
    """(rgb [B,H,W,3], depth [B,H,W,1], alpha [B,H,W,1]) in the inputs' dtype."""
    g = means.shape[0]
    dtype = means.dtype
    scales = torch.exp(log_scales)
    rot = quaternion_rotation(rotations)
    sigma3 = rot @ torch.diag_embed(scales * scales) @ rot.transpose(1, 2)
    opacity = torch.sigmoid(opacity_logits)
    ys, xs = torch.meshgrid(
        torch.arange(height, dtype=dtype) + 0.5, torch.arange(width, dtype=dtype) + 0.5, indexing="ij"
    )
    xs = xs.reshape(-1, 1)
    ys = ys.reshape(-1, 1)
    ids = torch.arange(g)
    rgbs, depths, alphas = [], [], []
    for b in range(viewmats.shape[0]):
        rc = viewmats[b, :3, :3]
        t = viewmats[b, :3, 3]
        fx, fy = intrinsics[b, 0, 0], intrinsics[b, 1, 1]
        cx, cy = intrinsics[b, 0, 2], intrinsics[b, 1, 2]
        p = means @ rc.T + t
        px, py, pz = p.unbind(-1)
        iz = 1.0 / pz
        u = fx * px * iz + cx
        v = fy * py * iz + cy
        cam = rc @ sigma3 @ rc.T
        tan_x = 0.5 * width / fx
        tan_y = 0.5 * height / fy
        lim_xp = 0.3 * tan_x + (width - cx) / fx
        lim_xn = 0.3 * tan_x + cx / fx
        lim_yp = 0.3 * tan_y + (height - cy) / fy
        lim_yn = 0.3 * tan_y + cy / fy
        ctx = torch.maximum(torch.minimum(px * iz, lim_xp), -lim_xn)
        cty = torch.maximum(torch.minimum(py * iz, lim_yp), -lim_yn)
        clx, cly = pz * ctx, pz * cty
        j00, j11 = fx * iz, fy * iz
        j02 = -fx * clx * iz * iz
        j12 = -fy * cly * iz * iz
        c00, c01, c02 = cam[:, 0, 0], cam[:, 0, 1], cam[:, 0, 2]
        c11, c12, c22 = cam[:, 1, 1], cam[:, 1, 2], cam[:, 2, 2]
        a = j00 * j00 * c00 + 2 * j00 * j02 * c02 + j02 * j02 * c22 + covariance_epsilon
        bb = j00 * j11 * c01 + j00 * j12 * c02 + j02 * j11 * c12 + j02 * j12 * c22
        c = j11 * j11 * c11 + 2 * j11 * j12 * c12 + j12 * j12 * c22 + covariance_epsilon
        det = a * c - bb * bb
        with torch.no_grad():
            o = opacity.detach()
            ext = torch.sqrt(2.0 * torch.log(torch.clamp(o / ALPHA_THRESHOLD, min=1.0)))
            ext = torch.clamp(ext, max=support_sigma)
            rx = torch.ceil(ext * torch.sqrt(torch.clamp(a.detach(), min=0.0)))
            ry = torch.ceil(ext * torch.sqrt(torch.clamp(c.detach(), min=0.0)))
            ud, vd = u.detach(), v.detach()
            visible = (
                (o >= ALPHA_THRESHOLD)
                & (pz.detach() >= near_plane)
                & (pz.detach() <= far_plane)
                & (det.detach() > 0)
                & ~((rx <= 0) & (ry <= 0))
                & ~((ud + rx <= 0) | (vd + ry <= 0) | (ud - rx >= width) | (vd - ry >= height))
            )
        safe_det = torch.where(visible, det, torch.ones_like(det))
        con0, con1, con2 = c / safe_det, -bb / safe_det, a / safe_det
        if sh_degree < 0:
            colors = features[:, :3]
        else:
            k = (sh_degree + 1) ** 2
            dirs = p @ rc  # R^T p, the direction from the camera centre to the mean
            dirs = dirs / torch.linalg.norm(dirs, dim=-1, keepdim=True)
            coeffs = features[:, : k * 3].reshape(g, k, 3)
            colors = torch.clamp((sh_basis(dirs, sh_degree).unsqueeze(-1) * coeffs).sum(1) + 0.5, min=0.0)
        order = ids[visible][torch.argsort(pz.detach()[visible], stable=True)]
        dx = xs - u[order]
        dy = ys - v[order]
        power = -0.5 * (con0[order] * dx * dx + 2 * con1[order] * dx * dy + con2[order] * dy * dy)
        raw = opacity[order] * torch.exp(power)
        alpha = torch.clamp(raw, max=MAX_ALPHA)
        with torch.no_grad():
            valid = (power <= 0) & (power >= -20.0) & (alpha >= ALPHA_THRESHOLD)
            a0 = torch.where(valid, alpha, torch.zeros_like(alpha))
            t_excl = torch.cumprod(
                torch.cat([torch.ones_like(a0[:, :1]), 1.0 - a0[:, :-1]], dim=1), dim=1
            )
            stop = valid & (t_excl * (1.0 - a0) <= TRANSMITTANCE_THRESHOLD)
            keep = valid & (torch.cumsum(stop.to(torch.int64), dim=1) == 0)
        alpha = torch.where(keep, alpha, torch.zeros_like(alpha))
        one_minus = 1.0 - alpha
        t = torch.cumprod(torch.cat([torch.ones_like(alpha[:, :1]), one_minus[:, :-1]], dim=1), dim=1)
        w = alpha * t
        rgb = w @ colors[order]
        dep = w @ pz[order]
        acc = 1.0 - torch.prod(one_minus, dim=1)
        ok = acc > 1e-8
        depth = torch.where(ok, dep / torch.where(ok, acc, torch.ones_like(acc)), torch.full_like(acc, math.inf))
        rgbs.append(rgb.reshape(height, width, 3))
        depths.append(depth.reshape(height, width, 1))
        alphas.append(acc.reshape(height, width, 1))
    return torch.stack(rgbs), torch.stack(depths), torch.stack(alphas)


def weighted_loss(rgb, depth, alpha, weights):
    """Linear test loss sum(w_rgb rgb) + sum(w_d depth over finite depth) + sum(w_a alpha)."""
    wr, wd, wa = weights
    finite = torch.isfinite(depth)
    d = torch.where(finite, depth, torch.zeros_like(depth))
    return (wr * rgb).sum() + (wd * d).sum() + (wa * alpha).sum()
