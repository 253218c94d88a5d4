"""Where the reference's CUDA build and the oracle differ at full size, and why.

On the batched workload (1M Gaussians, features[0..2] as linear RGB, four of
the 64 cameras at 640x480) the reference's own CUDA build and the oracle
agree to 1e-4 on all but a small set of pixels (the golden record
tests/golden/camera_threshold_flips.npz, made on a B200 by
tests/golden/make_threshold_golden.py).  The reference evaluates its
compositor and projection with fast-math intrinsics (renderer_cuda.cu is
built with --use_fast_math; __expf, approximate division and contracted
products), the oracle and this library with IEEE round-to-nearest
operations, so the two evaluate the same equation a few ulp apart.  That
moves a pixel by more than rounding only where a discrete decision of the
equation sits within those few ulp of its threshold:

* a record's alpha o exp(power) against the 1/255 floor, or its power
  against the -20 cut (renderer_cuda.cu:2203-2271);
* a running transmittance against the 1e-4 stop;
* two blended records whose depths are a few ulp apart, whose order can
  swap (the sort key is the float bits of depth).

The oracle reports, per pixel, the relative distance of the closest such
decision (camera_oracle.c, vo_set_margin_output).  This test re-renders the
case with the oracle and checks that every pixel the reference moved by
more than 1e-4 has a decision within 1e-4 (relative) of its threshold, or a
pair of blended depths within 1e-6, while such near-threshold pixels are
rare in the frame as a whole (so the explanation is not vacuous).  On the
recorded case 182 of 1,228,800 pixels differ by more than 1e-4 (at most
0.0085), every one of them near a threshold, against about 4 % of all
pixels near one.
"""

from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).resolve().parent / "golden" / "camera_threshold_flips.npz"
DECISION_MARGIN = 1.0e-4
DEPTH_MARGIN = 1.0e-6


@pytest.fixture(scope="module")
def frame():
    if not GOLDEN.exists():
        pytest.skip("golden record not generated (tests/golden/make_threshold_golden.py on a CUDA machine)")
    from golden.make_threshold_golden import case, oracle_frame

    golden = dict(np.load(GOLDEN))
    scene, rig = case()
    assert tuple(golden["cameras"]) == (0, 16, 32, 48)
    return golden, oracle_frame(scene, rig)


def test_oracle_reproduces_the_recorded_frame(frame):
    golden, got = frame
    rgb = got.rgb.reshape(-1, 3)
    assert rgb.shape[0] == int(golden["pixels"])
    np.testing.assert_array_equal(rgb[golden["flagged"]], golden["oracle_rgb"])
    assert [got.visible, got.intersections] == golden["oracle_counters"].tolist()


def test_every_pixel_over_1e4_sits_on_a_decision_threshold(frame):
    golden, got = frame
    margins = got.margins.reshape(-1, 3)[golden["flagged"]]
    near = (np.minimum(margins[:, 0], margins[:, 1]) < DECISION_MARGIN) | (margins[:, 2] < DEPTH_MARGIN)
    unexplained = golden["flagged"][~near]
    assert unexplained.size == 0, (unexplained[:20], margins[~near][:20])
    # Everywhere else the two builds agree to 1e-4.
    assert float(golden["max_abs_elsewhere"]) <= 1e-4


def test_near_threshold_pixels_are_rare(frame):
    golden, got = frame
    margins = got.margins.reshape(-1, 3)
    near = (np.minimum(margins[:, 0], margins[:, 1]) < DECISION_MARGIN) | (margins[:, 2] < DEPTH_MARGIN)
    fraction = float(near.mean())
    flagged = int(golden["flagged"].size)
    # About one pixel in twenty-five sits this close to a decision (most of
    # them do not flip), so if the flipped pixels were unrelated to the
    # thresholds, all of them landing among the near ones would have
    # probability fraction ** flagged.
    assert 0.0 < fraction < 0.1, fraction
    assert flagged >= 50
    assert flagged * np.log10(fraction) < -50.0
