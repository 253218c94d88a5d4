"""Generate PLY-ingestion golden vectors from the reference's own loader.

Writes a small binary little-endian INRIA 3DGS PLY (tests/golden/ply_sh3.ply:
48 Gaussians with SH degree 3, a semantic_id property, one all-zero
quaternion and a few extreme activations), then runs the reference's
ply_loader.load_ply_to_gaussians and canonicalize_3dgs_scene
(src/isaacsim_gaussian_renderer/ply_loader.py) on it and stores both results
in tests/golden/ply_sh3.npz.  plyfile is not installed in this image, so a
minimal stand-in module with the one call the loader makes
(PlyData.read(path).elements[0][name] and .properties[i].name) is
registered first; it reads the file written here with numpy.

Usage: python tests/golden/make_ply_golden.py [--reference PATH]  (default: $VGR_REFERENCE_ROOT)
"""

from __future__ import annotations

import argparse
import os
import sys
import types
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
COUNT = 48
REST = 45


def property_names() -> list[str]:
    names = ["x", "y", "z", "nx", "ny", "nz", "f_dc_0", "f_dc_1", "f_dc_2"]
    names += [f"f_rest_{i}" for i in range(REST)]
    names += ["opacity", "scale_0", "scale_1", "scale_2", "rot_0", "rot_1", "rot_2", "rot_3"]
    return names


def write_ply(path: Path) -> None:
    rng = np.random.default_rng(2026)
    names = property_names()
    dtype = np.dtype([(n, "<f4") for n in names] + [("semantic_id", "<i4")])
    rows = np.zeros(COUNT, dtype=dtype)
    for n in names:
        rows[n] = rng.normal(0.0, 1.0, COUNT).astype(np.float32)
    rows["opacity"][:4] = [-30.0, 30.0, 0.0, 8.0]
    rows["scale_0"][4] = -12.0
    for n in ("rot_0", "rot_1", "rot_2", "rot_3"):
        rows[n][5] = 0.0
    rows["f_dc_0"][6] = 10.0
    rows["f_dc_1"][6] = -10.0
    rows["semantic_id"] = rng.integers(0, 1000, COUNT).astype(np.int32)
    header = ["ply", "format binary_little_endian 1.0", "comment written by make_ply_golden.py",
              f"element vertex {COUNT}"]
    header += [f"property float {n}" for n in names] + ["property int semantic_id", "end_header"]
    with path.open("wb") as f:
        f.write(("\n".join(header) + "\n").encode("ascii"))
        f.write(rows.tobytes())


def plyfile_stand_in() -> types.ModuleType:
    module = types.ModuleType("plyfile")

    class _Element:
        def __init__(self, data: np.ndarray):
            self._data = data
            self.properties = [types.SimpleNamespace(name=n) for n in data.dtype.names]

        def __len__(self) -> int:
            return len(self._data)

        def __getitem__(self, name: str) -> np.ndarray:
            return self._data[name]

    class PlyData:
        @staticmethod
        def read(path: str):
            raw = Path(path).read_bytes()
            end = raw.index(b"end_header\n") + len(b"end_header\n")
            fields = []
            count = 0
            for line in raw[:end].decode("ascii").splitlines():
                parts = line.split()
                if parts[:2] == ["element", "vertex"]:
                    count = int(parts[2])
                elif parts and parts[0] == "property":
                    fields.append((parts[2], {"float": "<f4", "int": "<i4"}[parts[1]]))
            data = np.frombuffer(raw[end:], dtype=np.dtype(fields), count=count)
            return types.SimpleNamespace(elements=[_Element(data)])

    module.PlyData = PlyData
    return module


def main() -> None:
    parser = argparse.ArgumentParser()
    parser.add_argument("--reference", default=os.environ.get("VGR_REFERENCE_ROOT"), required="VGR_REFERENCE_ROOT" not in os.environ)
    args = parser.parse_args()
    ply = HERE / "ply_sh3.ply"
    write_ply(ply)
    sys.modules["plyfile"] = plyfile_stand_in()
    sys.path.insert(0, str(Path(args.reference) / "src"))
    from isaacsim_gaussian_renderer import ply_loader  # noqa: E402

    raw = ply_loader.load_ply_to_gaussians(ply)
    canonical = ply_loader.canonicalize_3dgs_scene(raw, device="cpu")
    out = {}
    for prefix, scene in (("raw", raw), ("canonical", canonical)):
        for name in ("means", "scales", "rotations", "opacities", "features", "semantic_ids"):
            out[f"{prefix}_{name}"] = getattr(scene, name).numpy()
    out["property_names"] = np.array(ply_loader.ply_vertex_property_names(ply))
    np.savez_compressed(HERE / "ply_sh3.npz", **out)
    print("wrote", ply, HERE / "ply_sh3.npz")


if __name__ == "__main__":
    main()
