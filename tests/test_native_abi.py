"""The C-ABI library loads without a GPU and exports every declared symbol."""

from __future__ import annotations

import re
from pathlib import Path

import pytest

from vgr_b200 import _native

HEADER_DIR = Path(__file__).resolve().parents[1] / "include"
DECL = re.compile(r"^\s*(?:const\s+)?[A-Za-z_][\w]*\s*\*?\s*(vgr_\w+)\s*\(", re.MULTILINE)


def declared_symbols() -> list[str]:
    names: list[str] = []
    for header in sorted(HEADER_DIR.glob("*.h")):
        names.extend(DECL.findall(header.read_text()))
    return sorted(set(names))


def test_header_declares_entry_points():
    names = declared_symbols()
    for expected in (
        "vgr_render",
        "vgr_sort_temp_bytes",
        "vgr_radix_sort_double_buffer_temp_bytes",
        "vgr_precompute_covariances",
        "vgr_prepare_chunked_active_ids",
        "vgr_aggregate_chunk_counters",
    ):
        assert expected in names


def test_library_exports_every_declared_symbol():
    lib = _native.load_library()
    missing = [name for name in declared_symbols() if not hasattr(lib, name)]
    assert not missing, missing
    typed = {name for name, _, _ in _native.CAMERA_SIGNATURES}
    from vgr_b200 import _native_signatures

    typed |= {name for name, _, _ in _native_signatures.extra_signatures()}
    assert set(declared_symbols()) <= typed


def test_version_and_scratch_queries_run_on_host():
    lib = _native.load_library()
    assert b"sm_100a" in lib.vgr_version()
    small = lib.vgr_render_scratch_bytes(1000, 10_000, 256, 1)
    large = lib.vgr_render_scratch_bytes(1_000_000, 64_000_000, 76_800, 64)
    assert 0 < small < large
    assert small % 256 == 0
    # The drop-in temp-bytes queries include the projected-record region.
    assert lib.vgr_radix_sort_double_buffer_temp_bytes(1000, 256) >= 1000 * _native.RECORD_BYTES


def test_static_scratch_limit_is_the_largest_fitting_camera_count():
    lib = _native.load_library()
    limit = lib.vgr_static_scratch_max_cameras()
    static_bytes = 16 << 20
    # 176 bytes per active camera (plan, projection constants, tile prefix)
    # plus a constant part of about 9 KB.
    assert 95_000 < limit < 96_000
    assert lib.vgr_render_scratch_bytes(1, 0, 1, limit) <= static_bytes
    assert lib.vgr_render_scratch_bytes(1, 0, 1, limit + 1) > static_bytes


@pytest.mark.parametrize(
    "items,segments,message",
    [
        (0, 1, "num_items must be positive"),
        (1, 0, "num_segments must be positive"),
        (2**31, 1, "INT_MAX intersections"),
    ],
)
def test_scratch_query_errors_match_reference_messages(items, segments, message):
    lib = _native.load_library()
    assert lib.vgr_sort_temp_bytes(items, segments) < 0
    assert message in _native.last_error()
