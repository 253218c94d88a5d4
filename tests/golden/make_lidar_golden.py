"""Generate LiDAR golden vectors from the reference's own CPU oracle.

Imports experiments/lidar_cpu_oracle.py from the reference checkout (pure
NumPy, float64) and stores, for each case, the inputs and its outputs in
tests/golden/lidar_<case>.npz.  The cases restate the reference's oracle
known-answer tests (tests/test_lidar_oracle.py:35-223: two-return clustering,
semantic and intensity weighting, no-hit contract, WXYZ rotation and
transform equivariance, near/far boundaries, grazing and thin surfaces,
batch/active subsets with scene transforms) and add randomized scenes on the
reference's randomized-oracle seeds (731, 2027, 99173, 104729) with a mix of
planar and non-planar Gaussians.

Usage: python tests/golden/make_lidar_golden.py [--reference PATH]  (default: $VGR_REFERENCE_ROOT)
"""

from __future__ import annotations

import argparse
import os
import math
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def make_scene(depths, *, semantics=None, reflectivity=None, rotation=None):
    count = len(depths)
    return {
        "means": np.array([[d, 0.0, 0.0] for d in depths], dtype=np.float64),
        "scales": np.array([[0.01, 1.0, 1.0]] * count, dtype=np.float64),
        "rotations": np.array([rotation if rotation is not None else [1.0, 0.0, 0.0, 0.0]] * count),
        "opacities": np.ones(count, dtype=np.float64),
        "semantic_ids": np.array(semantics or list(range(count)), dtype=np.int64),
        "reflectivity": None if reflectivity is None else np.array(reflectivity, dtype=np.float64),
    }


def identity(batch):
    return np.repeat(np.eye(4)[None], batch, axis=0)


def random_scene(seed: int, count: int):
    rng = np.random.default_rng(seed)
    means = np.c_[rng.uniform(2.0, 12.0, count), rng.normal(0.0, 0.8, (count, 2))]
    scales = np.exp(rng.normal(-1.5, 0.6, (count, 3)))
    planar = rng.random(count) < 0.7
    axis = rng.integers(0, 3, count)
    scales[planar, axis[planar]] *= 0.05
    quats = rng.normal(size=(count, 4))
    quats /= np.linalg.norm(quats, axis=1, keepdims=True)
    scene = {
        "means": means,
        "scales": scales,
        "rotations": quats,
        "opacities": rng.uniform(0.05, 1.0, count),
        "semantic_ids": rng.integers(0, 6, count).astype(np.int64),
        "reflectivity": rng.uniform(0.1, 0.9, count),
        "surface_confidence": rng.uniform(0.5, 1.0, count),
    }
    rays = rng.normal(size=(64, 3))
    rays[:, 0] = np.abs(rays[:, 0]) + 0.8
    rays /= np.linalg.norm(rays, axis=1, keepdims=True)
    sensors = identity(2)
    sensors[1, :3, 3] = [0.3, -0.2, 0.1]
    return {5: scene}, rays, sensors, np.array([5, 5])


def cases():
    angle = math.radians(30.0)
    angled = np.array([math.cos(angle), math.sin(angle), 0.0])
    out = {}
    out["two_returns"] = dict(
        scenes={4: make_scene([5.0, 5.01, 8.0], semantics=[9, 3, 11], reflectivity=[0.2, 0.6, 0.8])},
        rays=np.array([[1.0, 0.0, 0.0], [0.0, 1.0, 0.0]]),
        times=np.array([0, 125]),
        sensors=identity(1),
        scene_ids=np.array([4]),
        kwargs=dict(returns=2),
    )
    half = math.sqrt(0.5)
    rot_scene = make_scene([0.0], semantics=[5], rotation=np.array([half, 0.0, 0.0, half]))
    rot_scene["means"][0] = [0.0, 5.0, 0.0]
    moved = identity(2)
    moved[1, :3, 3] = [3.0, -2.0, 1.0]
    out["rotation_translation"] = dict(
        scenes={1: rot_scene},
        rays=np.array([[0.0, 1.0, 0.0]]),
        times=np.array([9]),
        sensors=moved,
        scene_ids=np.array([1, 1]),
        kwargs=dict(scene_to_world=moved.copy()),
    )
    boundary = {
        1: make_scene([0.05], semantics=[1]),
        2: make_scene([200.0], semantics=[2]),
        3: make_scene([0.049], semantics=[3]),
        4: make_scene([200.001], semantics=[4]),
        5: make_scene([5.0], semantics=[5]),
        6: make_scene([0.0], semantics=[6], rotation=np.array([math.cos(angle / 2), 0, 0, math.sin(angle / 2)])),
        7: make_scene([4.0], semantics=[7]),
        8: make_scene([4.0], semantics=[8]),
    }
    boundary[6]["means"][0] = 5.0 * angled
    boundary[7]["means"][0] = [4.0, 0.05, 0.0]
    boundary[7]["scales"][0] = [0.01, 0.06, 0.5]
    boundary[8]["scales"][0] = [0.5, 1.0, 1.0]
    out["boundaries_grazing_thin"] = dict(
        scenes=boundary,
        rays=np.array([[1, 0, 0], [1, 0, 0], [1, 0, 0], [1, 0, 0], [0, 1, 0], angled, [1, 0, 0], [1, 0, 0]], dtype=np.float64),
        times=np.arange(8),
        sensors=identity(8),
        scene_ids=np.arange(1, 9),
        kwargs={},
    )
    xforms = identity(3)
    xforms[2, 0, 3] = 2.0
    out["batch_active_transforms"] = dict(
        scenes={2: make_scene([4.0], semantics=[2]), 8: make_scene([7.0], semantics=[8])},
        rays=np.array([[1.0, 0.0, 0.0]]),
        times=np.array([0]),
        sensors=identity(3),
        scene_ids=np.array([2, 8, 2]),
        kwargs=dict(scene_to_world=xforms, active_sensor_ids=np.array([0, 2])),
    )
    for seed in (731, 2027, 99173, 104729):
        scenes, rays, sensors, ids = random_scene(seed, 400)
        out[f"random_{seed}"] = dict(
            scenes=scenes, rays=rays, times=np.arange(rays.shape[0]) * 10, sensors=sensors,
            scene_ids=ids, kwargs=dict(returns=2),
        )
    return out


def save(name: str, case: dict, result: dict) -> None:
    arrays = {
        "rays": case["rays"], "times": case["times"], "sensors": case["sensors"],
        "scene_ids": case["scene_ids"],
        "returns": np.int64(case["kwargs"].get("returns", 1)),
        "scene_keys": np.array(list(case["scenes"]), dtype=np.int64),
    }
    if "scene_to_world" in case["kwargs"]:
        arrays["scene_to_world"] = case["kwargs"]["scene_to_world"]
    if "active_sensor_ids" in case["kwargs"]:
        arrays["active_sensor_ids"] = case["kwargs"]["active_sensor_ids"]
    for sid, scene in case["scenes"].items():
        for key, value in scene.items():
            if value is not None:
                arrays[f"scene{sid}_{key}"] = value
    for key, value in result.items():
        arrays[f"out_{key}"] = value
    np.savez_compressed(HERE / f"lidar_{name}.npz", **arrays)


def main() -> None:
    parser = argparse.ArgumentParser()
    parser.add_argument("--reference", type=Path, default=os.environ.get("VGR_REFERENCE_ROOT"), required="VGR_REFERENCE_ROOT" not in os.environ)
    args = parser.parse_args()
    sys.path.insert(0, str(args.reference))
    from experiments.lidar_cpu_oracle import render_lidar_oracle

    for name, case in cases().items():
        result = render_lidar_oracle(
            case["scenes"], case["rays"], case["times"], case["sensors"], case["scene_ids"],
            **case["kwargs"],
        )
        save(name, case, result)
        print(name, "valid returns:", int(np.asarray(result["valid"]).sum()))


if __name__ == "__main__":
    main()
