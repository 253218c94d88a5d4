"""The CPU LiDAR oracle against the reference's own oracle (no GPU).

Golden vectors come from the reference's experiments/lidar_cpu_oracle.py
(tests/golden/make_lidar_golden.py); the known answers restate
tests/test_lidar_oracle.py:35-223 of the reference.
"""

from __future__ import annotations

import numpy as np
import pytest

from golden import lidar_cases
from oracle import lidar as ol


@pytest.mark.parametrize("name", lidar_cases.names())
def test_oracle_matches_reference_golden(name):
    case = lidar_cases.load(name)
    got = ol.render(case["scenes"], case["rays"], case["times"], case["sensors"], case["scene_ids"], **case["kwargs"])
    want = case["expected"]
    for key in ("valid", "semantic_id", "return_count", "time_offset_ns"):
        np.testing.assert_array_equal(got[key], want[key], err_msg=key)
    for key in ("range_m", "intensity", "position_world_m"):
        np.testing.assert_allclose(got[key], want[key], rtol=0, atol=1e-9, err_msg=key)


def test_known_answers_two_returns_and_no_hit():
    case = lidar_cases.load("two_returns")
    got = ol.render(case["scenes"], case["rays"], case["times"], case["sensors"], case["scene_ids"], **case["kwargs"])
    assert got["valid"][0, 0].tolist() == [True, True]
    np.testing.assert_allclose(got["range_m"][0, 0], [5.005, 8.0], atol=1e-12)
    assert got["semantic_id"][0, 0].tolist() == [3, 11]
    np.testing.assert_allclose(got["intensity"][0, 0], [0.4, 0.8], atol=1e-12)
    assert got["return_count"][0, 0] == 2
    assert not got["valid"][0, 1].any()
    assert np.isinf(got["range_m"][0, 1]).all()
    assert (got["semantic_id"][0, 1] == -1).all()


def test_known_answers_boundaries():
    case = lidar_cases.load("boundaries_grazing_thin")
    got = ol.render(case["scenes"], case["rays"], case["times"], case["sensors"], case["scene_ids"], **case["kwargs"])
    selected = got["valid"][np.arange(8), np.arange(8), 0]
    assert selected.tolist() == [True, True, False, False, False, True, True, False]
    np.testing.assert_allclose(
        got["range_m"][[0, 1, 5, 6], [0, 1, 5, 6], 0], [0.05, 200.0, 5.0, 4.0], atol=1e-10
    )


def test_permutation_invariance():
    case = lidar_cases.load("random_731")
    base = ol.render(case["scenes"], case["rays"], case["times"], case["sensors"], case["scene_ids"], **case["kwargs"])
    rng = np.random.default_rng(5)
    scene = case["scenes"][5]
    perm = rng.permutation(scene["means"].shape[0])
    permuted = {5: {k: None if v is None else v[perm] for k, v in scene.items()}}
    got = ol.render(permuted, case["rays"], case["times"], case["sensors"], case["scene_ids"], **case["kwargs"])
    np.testing.assert_array_equal(got["valid"], base["valid"])
    np.testing.assert_array_equal(got["semantic_id"], base["semantic_id"])
    np.testing.assert_allclose(got["range_m"], base["range_m"], rtol=0, atol=1e-12)
