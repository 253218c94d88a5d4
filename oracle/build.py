"""Build the CPU parity oracles (test infrastructure only).

  liboracle_camera.so  <- oracle/camera_oracle.c (gcc, IEEE float, no contraction)
  liboracle_lidar.so   <- oracle/lidar_oracle.c (gcc, float64)

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg load
these libraries; the renderer itself never does.
"""

from __future__ import annotations

import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
FLAGS = [
    "-O3",
    "-std=c11",
    "-ffp-contract=off",
    "-fno-fast-math",
    "-fno-math-errno",
    "-mfma",
    "-fopenmp",
    "-fPIC",
    "-shared",
]


def _stale(target: Path, source: Path) -> bool:
    return not target.exists() or source.stat().st_mtime > target.stat().st_mtime


def build(force: bool = False) -> list[Path]:
    outputs = []
    for source, target in (
        (HERE / "camera_oracle.c", HERE / "liboracle_camera.so"),
        (HERE / "lidar_oracle.c", HERE / "liboracle_lidar.so"),
    ):
        if force or _stale(target, source):
            cmd = ["gcc", *FLAGS, str(source), "-o", str(target), "-lm"]
            result = subprocess.run(cmd, capture_output=True, text=True)
            if result.returncode != 0:
                sys.stderr.write(result.stdout + result.stderr)
                raise RuntimeError(f"oracle build failed for {source.name}")
        outputs.append(target)
    return outputs


if __name__ == "__main__":
    for path in build(force="--force" in sys.argv):
        print(path)
