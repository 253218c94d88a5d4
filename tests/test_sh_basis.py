"""The spherical-harmonics colour basis against its mathematical definition.

The reference renders features[0..2] as linear RGB only, and gsplat (whose
basis the SH colour mode follows) is not installed, so nothing of theirs can
pin the degree-1..3 evaluation.  This test pins it to mathematics instead:
the real spherical harmonics built from scipy's complex Y_l^m (which carry
the Condon-Shortley phase), Y_lm = sqrt(2) (-1)^m Re Y_l^m for m > 0,
sqrt(2) (-1)^m Im Y_l^|m| for m < 0, Y_l0 for m = 0, in the axis convention
z = cos(polar), x = sin(polar) cos(azimuth), y = sin(polar) sin(azimuth).
The 3D Gaussian Splatting basis is that one with the phase (-1)^m kept, at
index k = l^2 + l + m of the coefficient rows.  For each basis function and
each of 40 view directions the oracle renders one Gaussian at the origin
from a camera at -4 d; the centre pixel's colour is alpha (0.3 Y_k(d) + 0.5)
with only coefficient k set, so Y_k(d) is read back from the image.  The GPU
path equals the oracle bit for bit in the parity tests, so this pins both.
Also checked: the read-back basis is orthonormal under an equal-weight
quadrature of the sphere on a 600-point Fibonacci lattice (which integrates
the degree <= 6 products to about 3e-3).
"""

from __future__ import annotations

import math

import numpy as np
import scipy.special as sp
import torch

from oracle import camera as oc
from vgr_b200.workloads import look_at_viewmats, pinhole

DIRECTIONS = 40
SIZE = 9
SCALE = 0.3


def _directions(count: int = DIRECTIONS) -> np.ndarray:
    """A Fibonacci lattice of unit directions whose poles lie on the y axis
    (the look-at helper's up vector), so no direction is parallel to it."""
    k = np.arange(count) + 0.5
    polar = np.arccos(1.0 - 2.0 * k / count)
    azimuth = math.pi * (1.0 + 5.0 ** 0.5) * k
    return np.stack((np.sin(polar) * np.cos(azimuth), np.cos(polar), np.sin(polar) * np.sin(azimuth)), axis=1)


def _expected(d: np.ndarray) -> np.ndarray:
    """[N, 16] Gaussian-splatting basis values at unit directions d."""
    polar = np.arccos(np.clip(d[:, 2], -1.0, 1.0))
    azimuth = np.arctan2(d[:, 1], d[:, 0])
    out = np.zeros((d.shape[0], 16))
    for l in range(4):
        for m in range(-l, l + 1):
            y = sp.sph_harm_y(l, abs(m), polar, azimuth)
            if m > 0:
                real = math.sqrt(2.0) * (-1) ** m * y.real
            elif m < 0:
                real = math.sqrt(2.0) * (-1) ** m * y.imag
            else:
                real = y.real
            out[:, l * l + l + m] = (-1) ** m * real
    return out


def _read_back(d: np.ndarray) -> np.ndarray:
    """[N, 16] basis values recovered from oracle renders."""
    n = d.shape[0]
    eyes = torch.from_numpy(-4.0 * d)
    view = look_at_viewmats(eyes, torch.zeros((n, 3), dtype=torch.float64)).numpy().astype(np.float32)
    intr = pinhole(n, 8.0, 8.0, SIZE / 2.0, SIZE / 2.0).numpy()
    cov = oc.precompute_covariances(np.full((1, 3), 0.5, np.float32), np.array([[1.0, 0.0, 0.0, 0.0]], np.float32))
    got = np.zeros((n, 16))
    for first in range(0, 16, 3):
        feats = np.zeros((1, 48), np.float32)
        ks = list(range(first, min(first + 3, 16)))
        for ch, k in enumerate(ks):
            feats[0, 3 * k + ch] = SCALE
        res = oc.render(
            means=np.zeros((1, 3), np.float32), covariances=cov, opacities=np.array([0.5], np.float32),
            features=feats, semantic_ids=np.zeros(1, np.int64), registered_scene_ids=[0], scene_offsets=[0, 1],
            viewmats=view, intrinsics=intr, camera_scene_ids=[0] * n, height=SIZE, width=SIZE, sh_degree=3,
            near_plane=0.01, far_plane=100.0, tile_size=16,
        )
        centre = SIZE // 2
        alpha = res.alpha[:, centre, centre, 0].astype(np.float64)
        for ch, k in enumerate(ks):
            colour = res.rgb[:, centre, centre, ch].astype(np.float64) / alpha
            got[:, k] = (colour - 0.5) / SCALE
    return got


def test_sh_basis_matches_the_real_spherical_harmonics():
    d = _directions()
    got = _read_back(d)
    want = _expected(d)
    assert np.max(np.abs(got - want)) < 2e-6, np.max(np.abs(got - want))


def test_read_back_basis_is_orthonormal():
    d = _directions(600)
    got = _read_back(d)
    gram = got.T @ got * (4.0 * math.pi / d.shape[0])
    assert np.max(np.abs(gram - np.eye(16))) < 1e-2
