"""Constructor contracts of CustomCudaBackend that need no GPU: the mode
combinations the reference accepts or rejects (cuda_backend.py:127-200)."""

from __future__ import annotations

import pytest

from vgr_b200 import CustomCudaBackend


def test_dense_and_exact_ray_modes_are_accepted():
    dense = CustomCudaBackend(tile_size=1)
    assert dense.bin_tile_size == 16
    compact = CustomCudaBackend(tile_size=1, compact_projection_cache=True, deterministic=False)
    assert compact.compact_projection_cache
    ray = CustomCudaBackend(tile_size=16, ray_gaussian_evaluation=True)
    assert ray.ray_gaussian_evaluation and ray.bin_tile_size == 32
    assert CustomCudaBackend(tile_size=8, ray_gaussian_evaluation=True).bin_tile_size == 8


@pytest.mark.parametrize(
    "kwargs, message",
    [
        ({"tile_size": 2}, "tile_size=2"),
        ({"tile_size": 3}, "power of two"),
        ({"tile_size": 32}, "power of two"),
        ({"tile_size": 8, "compact_projection_cache": True}, "requires tile_size=1"),
        ({"tile_size": 1, "ray_gaussian_evaluation": True}, "screen-space"),
        ({"rasterize_mode": "antialiased", "ray_gaussian_evaluation": True}, "incompatible"),
        ({"materialize_projected_records": True}, "requires compact_projection_cache"),
    ],
)
def test_rejected_combinations(kwargs, message):
    with pytest.raises(ValueError, match=message):
        CustomCudaBackend(**kwargs)


def test_mode_setters_keep_the_combination_rules():
    backend = CustomCudaBackend(tile_size=16)
    backend.ray_gaussian_evaluation = True
    with pytest.raises(ValueError, match="incompatible"):
        backend.rasterize_mode = "antialiased"
    backend.ray_gaussian_evaluation = False
    backend.rasterize_mode = "antialiased"
    with pytest.raises(ValueError, match="incompatible"):
        backend.ray_gaussian_evaluation = True
    dense = CustomCudaBackend(tile_size=1)
    with pytest.raises(ValueError, match="screen-space"):
        dense.ray_gaussian_evaluation = True
