"""Entry points of libvgr_b200.so beyond the camera path (filled as added)."""

from __future__ import annotations


def extra_signatures() -> list[tuple[str, object, list[object]]]:
    return []
