"""Generate hybrid-compositor golden vectors from the reference's own function.

Imports src/isaacsim_gaussian_renderer/hybrid_compositor.py from the
reference checkout (pure torch) and stores random Gaussian and mesh layers
(including empty pixels, NaN/inf alpha and depth, alpha below the threshold
and near-equal depths) with the reference's composite in
tests/golden/hybrid_composite.npz.

Usage: python tests/golden/make_hybrid_golden.py [--reference PATH]  (default: $VGR_REFERENCE_ROOT)
"""

from __future__ import annotations

import argparse
import os
import sys
from pathlib import Path

import numpy as np
import torch

HERE = Path(__file__).resolve().parent


def layers(seed: int):
    gen = torch.Generator().manual_seed(seed)
    shape = (2, 9, 11)
    out = {}
    for name in ("gaussian", "mesh"):
        rgb = torch.rand((*shape, 3), generator=gen)
        alpha = torch.rand((*shape, 1), generator=gen)
        depth = torch.rand((*shape, 1), generator=gen) * 10 + 0.1
        flat_a = alpha.view(-1)
        flat_d = depth.view(-1)
        flat_a[::7] = 0.0
        flat_a[3::11] = 5e-5
        flat_a[5::13] = float("nan")
        flat_d[6::17] = float("inf")
        flat_d[8::19] = float("nan")
        out[name] = (rgb, alpha, depth)
    # near-equal depths around the epsilon
    g_d = out["gaussian"][2].view(-1)
    m_d = out["mesh"][2].view(-1)
    m_d[1::9] = g_d[1::9] - 5e-5
    m_d[2::9] = g_d[2::9] - 2e-4
    return out


def main() -> None:
    parser = argparse.ArgumentParser()
    parser.add_argument("--reference", default=os.environ.get("VGR_REFERENCE_ROOT"), required="VGR_REFERENCE_ROOT" not in os.environ)
    args = parser.parse_args()
    # Load the module file alone: the package's __init__ imports optional
    # dependencies (plyfile) that this image lacks.
    import importlib.util

    path = Path(args.reference) / "src" / "isaacsim_gaussian_renderer" / "hybrid_compositor.py"
    spec = importlib.util.spec_from_file_location("reference_hybrid_compositor", path)
    module = importlib.util.module_from_spec(spec)
    sys.modules[spec.name] = module
    spec.loader.exec_module(module)
    composite_gaussian_and_mesh = module.composite_gaussian_and_mesh

    data = {}
    for case, (seed, kwargs) in enumerate(((1, {}), (2, {"min_alpha": 0.3, "depth_epsilon": 0.0}))):
        ls = layers(seed)
        res = composite_gaussian_and_mesh(*ls["gaussian"], *ls["mesh"], **kwargs)
        for name, (rgb, alpha, depth) in ls.items():
            data[f"c{case}_{name}_rgb"] = rgb.numpy()
            data[f"c{case}_{name}_alpha"] = alpha.numpy()
            data[f"c{case}_{name}_depth"] = depth.numpy()
        data[f"c{case}_min_alpha"] = np.float64(kwargs.get("min_alpha", 1.0e-4))
        data[f"c{case}_depth_epsilon"] = np.float64(kwargs.get("depth_epsilon", 1.0e-4))
        for field in ("rgb", "alpha", "depth", "mesh_in_front"):
            data[f"c{case}_out_{field}"] = getattr(res, field).numpy()
    np.savez_compressed(HERE / "hybrid_composite.npz", **data)
    print("wrote", HERE / "hybrid_composite.npz")


if __name__ == "__main__":
    main()
