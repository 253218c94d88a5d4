"""INRIA 3D Gaussian Splatting PLY ingestion.

Counterpart of src/isaacsim_gaussian_renderer/ply_loader.py.  The header is
read on the host (it is a few hundred bytes of ASCII); the vertex body is
copied to the device as raw bytes and one CUDA kernel
(``vgr_ply_canonicalize``) reads every packed row at the header's byte
offsets and writes the renderer-ready canonical tensors (exp scales, sigmoid
opacity, normalised WXYZ quaternion, DC -> linear RGB, f_rest reordered to
coefficient-major), replacing the reference's plyfile parse, numpy stacking
and torch activation passes.  ``load_ply_to_gaussians`` keeps the
reference's raw host form.
"""

from __future__ import annotations

from dataclasses import dataclass
from pathlib import Path

import numpy as np
import torch

from . import _native
from .scene import GaussianScene

SH_C0 = 0.28209479177387814

_PLY_TYPES = {
    "char": (0, "i1"), "int8": (0, "i1"),
    "uchar": (1, "u1"), "uint8": (1, "u1"),
    "short": (2, "i2"), "int16": (2, "i2"),
    "ushort": (3, "u2"), "uint16": (3, "u2"),
    "int": (4, "i4"), "int32": (4, "i4"),
    "uint": (5, "u4"), "uint32": (5, "u4"),
    "int64": (6, "i8"), "long": (6, "i8"),
    "float": (7, "f4"), "float32": (7, "f4"),
    "double": (8, "f8"), "float64": (8, "f8"),
}
_ROLES = {"x": 0, "y": 1, "z": 2, "scale_0": 3, "scale_1": 4, "scale_2": 5, "rot_0": 6, "rot_1": 7,
          "rot_2": 8, "rot_3": 9, "opacity": 10, "f_dc_0": 11, "f_dc_1": 12, "f_dc_2": 13,
          "semantic_id": 14}
_REST0 = 15


@dataclass
class PlyVertexBlock:
    count: int
    properties: list[tuple[str, str]]  # (name, PLY type)
    body: np.ndarray                    # uint8 [count * row_bytes], packed little-endian rows
    row_bytes: int


def _parse_header(stream) -> tuple[str, int, list[tuple[str, str]]]:
    if stream.readline().strip() != b"ply":
        raise ValueError("PLY header must begin with the 'ply' magic line.")
    fmt = None
    count = None
    props: list[tuple[str, str]] = []
    in_vertex = False
    first_element = True
    while stream.tell() <= 1024 * 1024:
        raw = stream.readline()
        if not raw:
            break
        try:
            parts = raw.decode("ascii").strip().split()
        except UnicodeDecodeError as error:
            raise ValueError("PLY header is not ASCII.") from error
        if not parts or parts[0] in {"comment", "obj_info"}:
            continue
        if parts[0] == "format":
            fmt = parts[1]
        elif parts[0] == "end_header":
            if fmt is None or count is None:
                raise ValueError("PLY header lacks a format line or a vertex element.")
            return fmt, count, props
        elif parts[0] == "element":
            in_vertex = len(parts) >= 3 and parts[1] == "vertex"
            if in_vertex:
                if not first_element:
                    raise ValueError("the vertex element must come first in the PLY body.")
                count = int(parts[2])
            first_element = False
        elif parts[0] == "property" and in_vertex:
            if len(parts) == 3:
                if parts[1] not in _PLY_TYPES:
                    raise ValueError(f"Unsupported PLY property type {parts[1]!r}.")
                props.append((parts[2], parts[1]))
            elif len(parts) == 5 and parts[1] == "list":
                raise ValueError("list properties are not part of the 3DGS vertex layout.")
            else:
                raise ValueError(f"Malformed PLY property line: {raw!r}")
    raise ValueError("PLY header lacks end_header within the first MiB.")


def ply_vertex_property_names(path: str | Path) -> tuple[str, ...]:
    """Vertex property names from a PLY header, without loading its body."""
    with Path(path).open("rb") as stream:
        _, _, props = _parse_header(stream)
    return tuple(name for name, _ in props)


def read_ply_vertex_block(path: str | Path) -> PlyVertexBlock:
    """The vertex rows as packed little-endian bytes (binary files are read
    as they are; ASCII and big-endian bodies are converted)."""
    with Path(path).open("rb") as stream:
        fmt, count, props = _parse_header(stream)
        dtype = np.dtype([(name, "<" + _PLY_TYPES[t][1]) for name, t in props])
        if fmt == "binary_little_endian":
            body = np.fromfile(stream, dtype=np.uint8, count=count * dtype.itemsize)
        elif fmt == "binary_big_endian":
            big = np.fromfile(stream, dtype=dtype.newbyteorder(">"), count=count)
            body = big.astype(dtype).view(np.uint8)
        elif fmt == "ascii":
            table = np.loadtxt(stream, dtype=np.float64, max_rows=count, ndmin=2)
            rows = np.zeros(count, dtype=dtype)
            for i, (name, _) in enumerate(props):
                rows[name] = table[:, i]
            body = rows.view(np.uint8).reshape(-1)
        else:
            raise ValueError(f"Unsupported PLY format {fmt!r}.")
    if body.size != count * dtype.itemsize:
        raise ValueError("PLY body is shorter than its header declares.")
    return PlyVertexBlock(count=count, properties=props, body=np.ascontiguousarray(body),
                          row_bytes=dtype.itemsize)


def _layout(block: PlyVertexBlock) -> tuple[_native.VgrPlyLayout, int]:
    layout = _native.VgrPlyLayout()
    layout.row_bytes = block.row_bytes
    offsets = {}
    offset = 0
    for name, t in block.properties:
        offsets[name] = (offset, _PLY_TYPES[t][0])
        offset += np.dtype(_PLY_TYPES[t][1]).itemsize
    for name, role in _ROLES.items():
        if name == "semantic_id":
            continue
        if name not in offsets:
            raise ValueError(f"PLY vertex lacks the {name!r} property of the 3DGS layout.")
        layout.offsets[role], layout.types[role] = offsets[name]
    if "semantic_id" in offsets:
        layout.offsets[_ROLES["semantic_id"]], layout.types[_ROLES["semantic_id"]] = offsets["semantic_id"]
        layout.has_semantic = 1
    rest = sorted((n for n in offsets if n.startswith("f_rest_")), key=lambda n: int(n.rsplit("_", 1)[1]))
    if len(rest) % 3:
        raise ValueError(f"Expected an RGB-multiple number of f_rest fields, got {len(rest)}.")
    if _REST0 + len(rest) > _native.PLY_MAX_PROPERTIES:
        raise ValueError("too many f_rest fields (at most SH degree 3).")
    for i, name in enumerate(rest):
        layout.offsets[_REST0 + i], layout.types[_REST0 + i] = offsets[name]
    layout.rest_count = len(rest)
    return layout, 3 + len(rest)


def load_ply_to_canonical_gaussians(path: str | Path, *, device: torch.device | str = "cuda") -> GaussianScene:
    """Load a standard 3DGS PLY and return renderer-ready canonical tensors on
    ``device`` (ply_loader.py:138-144), activated on the GPU."""
    device = torch.device(device)
    if device.type != "cuda":
        raise ValueError("PLY canonicalisation runs on a CUDA device")
    block = read_ply_vertex_block(path)
    layout, width = _layout(block)
    count = block.count
    rows = torch.from_numpy(block.body).to(device)
    out = {
        "means": torch.empty((count, 3), dtype=torch.float32, device=device),
        "scales": torch.empty((count, 3), dtype=torch.float32, device=device),
        "rotations": torch.empty((count, 4), dtype=torch.float32, device=device),
        "opacities": torch.empty((count,), dtype=torch.float32, device=device),
        "features": torch.empty((count, width), dtype=torch.float32, device=device),
        "semantic_ids": torch.empty((count,), dtype=torch.int64, device=device),
    }
    lib = _native.load_library()
    with torch.cuda.device(device):
        _native.check(
            lib.vgr_ply_canonicalize(
                rows.data_ptr(), count, layout, out["means"].data_ptr(), out["scales"].data_ptr(),
                out["rotations"].data_ptr(), out["opacities"].data_ptr(), out["features"].data_ptr(),
                width, out["semantic_ids"].data_ptr(), torch.cuda.current_stream(device).cuda_stream,
            ),
            "ply_canonicalize",
        )
    return GaussianScene(**out)


def load_ply_to_gaussians(path: str | Path) -> GaussianScene:
    """Raw 3DGS parameters as CPU tensors (ply_loader.py:52-90): means,
    log-scales, raw quaternions, opacity logits, features = (f_dc, f_rest
    coefficient-major), semantic_id or zeros."""
    block = read_ply_vertex_block(path)
    dtype = np.dtype([(name, "<" + _PLY_TYPES[t][1]) for name, t in block.properties])
    rows = block.body.view(dtype)
    names = [n for n, _ in block.properties]

    def stack(cols: list[str]) -> np.ndarray:
        return np.stack([rows[c].astype(np.float32) for c in cols], axis=1)

    rest = sorted((n for n in names if n.startswith("f_rest_")), key=lambda n: int(n.rsplit("_", 1)[1]))
    if len(rest) % 3:
        raise ValueError(f"Expected an RGB-multiple number of f_rest fields, got {len(rest)}.")
    count = block.count
    sh0 = stack(["f_dc_0", "f_dc_1", "f_dc_2"])[:, None, :]
    shn = stack(rest).reshape(count, 3, len(rest) // 3).swapaxes(1, 2) if rest else np.zeros((count, 0, 3), np.float32)
    scales = sorted((n for n in names if n.startswith("scale_")), key=lambda n: int(n.rsplit("_", 1)[1]))
    rots = sorted((n for n in names if n.startswith("rot_")), key=lambda n: int(n.rsplit("_", 1)[1]))
    semantic = rows["semantic_id"].astype(np.int64) if "semantic_id" in names else np.zeros(count, np.int64)
    return GaussianScene(
        means=torch.from_numpy(np.ascontiguousarray(stack(["x", "y", "z"]))),
        scales=torch.from_numpy(np.ascontiguousarray(stack(scales))),
        rotations=torch.from_numpy(np.ascontiguousarray(stack(rots))),
        opacities=torch.from_numpy(np.ascontiguousarray(rows["opacity"].astype(np.float32))),
        features=torch.from_numpy(np.ascontiguousarray(np.concatenate((sh0, shn), axis=1).reshape(count, -1))),
        semantic_ids=torch.from_numpy(np.ascontiguousarray(semantic)),
    )
