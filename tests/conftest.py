"""Test configuration: the ``gpu`` marker and import paths.

The renderer package lives in ``vectorized-gaussian-renderer-public_b200/``
(a source directory like the reference's ``src/``); the CPU oracle in
``oracle/``.
"""

from __future__ import annotations

import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
PKG_ROOT = ROOT / "vectorized-gaussian-renderer-public_b200"
for path in (str(ROOT / "tests"), str(PKG_ROOT), str(ROOT)):
    if path not in sys.path:
        sys.path.insert(0, path)


def pytest_configure(config: pytest.Config) -> None:
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libvgr_b200.so")


def pytest_collection_modifyitems(config: pytest.Config, items: list[pytest.Item]) -> None:
    import torch

    if torch.cuda.is_available():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)
