"""Recipe: compile the reference's own camera and LiDAR extensions for sm_100a.

TEST INFRASTRUCTURE ONLY.  Builds, from the sources where they lie in the
read-only reference checkout (never copied into this repository),

  src/isaacsim_gaussian_renderer/native/renderer.cpp + renderer_cuda.cu
      -> oracle/_ref/vgr_reference_camera.so
  src/isaacsim_gaussian_renderer/native/lidar_renderer.cpp + lidar_renderer_cuda.cu
      -> oracle/_ref/vgr_reference_lidar.so

with the reference's own flags (camera: -O3 --use_fast_math -lineinfo,
native_loader.py:15-20; LiDAR: -O3 -lineinfo, lidar_native_loader.py) plus
-gencode arch=compute_100a,code=sm_100a.  The outputs are git-ignored and
travel to the GPU machine with the working tree, where
tests/golden/make_reference_golden.py runs them to produce golden vectors.

The checkout's location is the --reference argument, else the
VGR_REFERENCE_ROOT environment variable; without either nothing is built.

Usage: python oracle/build_ref.py [--reference /path/to/reference]
"""

from __future__ import annotations

import argparse
import os
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "_ref"


def reference_root() -> Path | None:
    """The reference checkout named by VGR_REFERENCE_ROOT, if it exists."""
    value = os.environ.get("VGR_REFERENCE_ROOT")
    if not value:
        return None
    path = Path(value)
    return path if path.exists() else None


NATIVE = Path("src/isaacsim_gaussian_renderer/native")
TARGETS = {
    "vgr_reference_camera": (
        ["renderer.cpp", "renderer_cuda.cu"],
        ["-O3", "--use_fast_math", "-lineinfo"],
    ),
    "vgr_reference_lidar": (
        ["lidar_renderer.cpp", "lidar_renderer_cuda.cu"],
        ["-O3", "-lineinfo"],
    ),
}


def build(reference: Path | None = None, optional: bool = False) -> list[Path]:
    reference = reference or reference_root()
    if reference is None:
        if optional:
            return []
        raise FileNotFoundError("set VGR_REFERENCE_ROOT or pass --reference")
    native = reference / NATIVE
    if not native.exists():
        if optional:
            return []
        raise FileNotFoundError(native)
    OUT.mkdir(parents=True, exist_ok=True)
    os.environ.setdefault("TORCH_CUDA_ARCH_LIST", "10.0")
    os.environ.setdefault("MAX_JOBS", str(os.cpu_count() or 4))
    from torch.utils.cpp_extension import load

    built = []
    for name, (sources, flags) in TARGETS.items():
        target = OUT / f"{name}.so"
        srcs = [native / s for s in sources]
        if target.exists() and all(s.stat().st_mtime <= target.stat().st_mtime for s in srcs):
            built.append(target)
            continue
        build_dir = OUT / f"build_{name}"
        build_dir.mkdir(parents=True, exist_ok=True)
        load(
            name=name,
            sources=[str(s) for s in srcs],
            build_directory=str(build_dir),
            extra_cflags=["-O3"],
            extra_cuda_cflags=[*flags, "-gencode", "arch=compute_100a,code=sm_100a"],
            verbose=False,
        )
        produced = build_dir / f"{name}.so"
        produced.replace(target)
        built.append(target)
    return built


def load_reference_module(name: str):
    """Import a built reference extension from oracle/_ref (GPU machine side)."""
    import importlib.machinery
    import importlib.util

    import torch  # noqa: F401  (loads libtorch for the extension)

    path = OUT / f"{name}.so"
    loader = importlib.machinery.ExtensionFileLoader(name, str(path))
    spec = importlib.util.spec_from_file_location(name, str(path), loader=loader)
    module = importlib.util.module_from_spec(spec)
    loader.exec_module(module)
    return module


if __name__ == "__main__":
    parser = argparse.ArgumentParser()
    parser.add_argument("--reference", type=Path, default=None)
    args = parser.parse_args()
    for path in build(args.reference):
        print(path)
