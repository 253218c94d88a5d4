"""Load the LiDAR golden fixtures written by make_lidar_golden.py."""

from __future__ import annotations

from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
SCENE_FIELDS = ("means", "scales", "rotations", "opacities", "semantic_ids", "reflectivity", "surface_confidence")


def names() -> list[str]:
    return sorted(p.stem[len("lidar_"):] for p in HERE.glob("lidar_*.npz"))


def load(name: str) -> dict:
    data = np.load(HERE / f"lidar_{name}.npz")
    scenes = {}
    for sid in data["scene_keys"].tolist():
        scene = {}
        for field in SCENE_FIELDS:
            key = f"scene{sid}_{field}"
            scene[field] = data[key] if key in data else None
        scenes[int(sid)] = scene
    kwargs = {"returns": int(data["returns"])}
    if "scene_to_world" in data:
        kwargs["scene_to_world"] = data["scene_to_world"]
    if "active_sensor_ids" in data:
        kwargs["active_sensor_ids"] = data["active_sensor_ids"]
    expected = {key[len("out_"):]: data[key] for key in data if key.startswith("out_")}
    return {
        "scenes": scenes,
        "rays": data["rays"],
        "times": data["times"],
        "sensors": data["sensors"],
        "scene_ids": data["scene_ids"],
        "kwargs": kwargs,
        "expected": expected,
    }
