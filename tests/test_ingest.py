"""Scene and camera ingestion against the reference's loader.

tests/golden/ply_sh3.{ply,npz} come from tests/golden/make_ply_golden.py,
which ran the reference's load_ply_to_gaussians and canonicalize_3dgs_scene
on the committed PLY.  Host parsing is checked on CPU; the CUDA
canonicalisation and camera conversion on the GPU.
"""

from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest
import torch

from vgr_b200.ply import load_ply_to_gaussians, ply_vertex_property_names, read_ply_vertex_block

GOLDEN = Path(__file__).resolve().parent / "golden"
PLY = GOLDEN / "ply_sh3.ply"


def _golden():
    return np.load(GOLDEN / "ply_sh3.npz")


def test_header_and_raw_load_match_reference():
    g = _golden()
    assert ply_vertex_property_names(PLY) == tuple(g["property_names"].tolist())
    raw = load_ply_to_gaussians(PLY)
    for name in ("means", "scales", "rotations", "opacities", "features", "semantic_ids"):
        np.testing.assert_array_equal(getattr(raw, name).numpy(), g[f"raw_{name}"], err_msg=name)


def test_malformed_ply_is_rejected(tmp_path):
    bad = tmp_path / "bad.ply"
    bad.write_bytes(b"plx\n")
    with pytest.raises(ValueError, match="magic"):
        ply_vertex_property_names(bad)
    rest = tmp_path / "rest.ply"
    header = ["ply", "format binary_little_endian 1.0", "element vertex 1"]
    header += [f"property float {n}" for n in ("x", "y", "z", "f_dc_0", "f_dc_1", "f_dc_2", "f_rest_0",
                                               "opacity", "scale_0", "scale_1", "scale_2",
                                               "rot_0", "rot_1", "rot_2", "rot_3")]
    rest.write_bytes(("\n".join(header + ["end_header"]) + "\n").encode() + np.zeros(15, "<f4").tobytes())
    with pytest.raises(ValueError, match="RGB-multiple"):
        load_ply_to_gaussians(rest)
    block = read_ply_vertex_block(rest)
    assert block.count == 1 and block.row_bytes == 60


@pytest.mark.gpu
def test_gpu_canonicalisation_matches_reference():
    from vgr_b200.ply import load_ply_to_canonical_gaussians

    g = _golden()
    scene = load_ply_to_canonical_gaussians(PLY, device="cuda")
    np.testing.assert_array_equal(scene.means.cpu().numpy(), g["canonical_means"])
    np.testing.assert_array_equal(scene.semantic_ids.cpu().numpy(), g["canonical_semantic_ids"])
    # exp / sigmoid / sqrt: CUDA's and torch-CPU's functions may differ by an ulp.
    np.testing.assert_allclose(scene.scales.cpu().numpy(), g["canonical_scales"], rtol=2e-6, atol=0)
    np.testing.assert_allclose(scene.opacities.cpu().numpy(), g["canonical_opacities"], rtol=2e-6, atol=1e-30)
    np.testing.assert_allclose(scene.rotations.cpu().numpy(), g["canonical_rotations"], rtol=2e-6, atol=1e-7)
    np.testing.assert_allclose(scene.features.cpu().numpy(), g["canonical_features"], rtol=2e-6, atol=1e-7)
    np.testing.assert_array_equal(scene.rotations[5].cpu().numpy(), [1.0, 0.0, 0.0, 0.0])


@pytest.mark.gpu
def test_gpu_world_to_opencv_matches_the_usd_convention():
    from vgr_b200.camera_ingest import world_to_opencv_viewmats

    gen = torch.Generator().manual_seed(4)
    n = 6
    q = torch.randn((n, 4), generator=gen, dtype=torch.float64)
    q = q / q.norm(dim=1, keepdim=True)
    w, x, y, z = q.unbind(1)
    rot = torch.stack([
        1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y),
        2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x),
        2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y),
    ], 1).reshape(n, 3, 3)
    world = torch.zeros((n, 4, 4), dtype=torch.float64)
    world[:, :3, :3] = rot.transpose(1, 2)  # USD row-vector: rows are the camera axes
    world[:, 3, :3] = torch.randn((n, 3), generator=gen, dtype=torch.float64) * 5
    world[:, 3, 3] = 1.0
    indices = torch.tensor([3, 0, 5, 1, 9, 2], dtype=torch.int32)
    viewmats = torch.full((6, 4, 4), -7.0)
    bad = world_to_opencv_viewmats(world.cuda(), v := viewmats.cuda(), indices.cuda())
    got = v.cpu()
    assert bad == 1  # index 9 is outside the 6 view matrices
    for i, out in enumerate(indices.tolist()):
        if out >= 6:
            continue
        r = world[i, :3, :3].float().clone()
        r[1] = -r[1]
        r[2] = -r[2]
        pos = world[i, 3, :3].float()
        want = torch.eye(4)
        want[:3, :3] = r
        want[:3, 3] = -(r @ pos)
        torch.testing.assert_close(got[out], want, rtol=1e-6, atol=1e-5)
    assert torch.all(got[4] == -7.0)  # no camera maps to row 4


@pytest.mark.gpu
@pytest.mark.parametrize("case", [0, 1])
def test_gpu_hybrid_composite_matches_reference(case):
    from vgr_b200.hybrid_compositor import composite_gaussian_and_mesh

    g = np.load(GOLDEN / "hybrid_composite.npz")
    t = {k: torch.from_numpy(g[f"c{case}_{k}"]).cuda() for k in (
        "gaussian_rgb", "gaussian_alpha", "gaussian_depth", "mesh_rgb", "mesh_alpha", "mesh_depth")}
    res = composite_gaussian_and_mesh(
        t["gaussian_rgb"], t["gaussian_alpha"], t["gaussian_depth"], t["mesh_rgb"], t["mesh_alpha"],
        t["mesh_depth"], min_alpha=float(g[f"c{case}_min_alpha"]), depth_epsilon=float(g[f"c{case}_depth_epsilon"]))
    for field in ("rgb", "alpha", "depth", "mesh_in_front"):
        np.testing.assert_array_equal(getattr(res, field).cpu().numpy(), g[f"c{case}_out_{field}"], err_msg=field)
