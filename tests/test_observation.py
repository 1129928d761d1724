"""Observation points and frames (host only): the custom-point, sphere-point and arc behaviour the
reference's unit tests pin (tests/test_observation.py:21-280); frames inferred from meshes are covered
by the golden fixtures of tests/test_frontend_golden.py."""
from __future__ import annotations

import numpy as np
import pytest

from hornlab_metal_bem_b200.config import ObservationConfig
from hornlab_metal_bem_b200.observation import ObservationFrame, build_observation_points

FRAME = ObservationFrame(axis=np.array([0.0, 0.0, 1.0]), origin=np.zeros(3), u=np.array([1.0, 0.0, 0.0]),
                         v=np.array([0.0, 1.0, 0.0]), mouth_center=np.array([0.0, 0.0, 1.0]),
                         source_center=np.zeros(3))


def test_sphere_points_validation():
    assert ObservationConfig(sphere_points=np.ones((5, 3))).sphere_points.shape == (5, 3)
    for bad in (np.zeros((4, 2)), np.zeros((0, 3)), np.zeros((3,))):
        with pytest.raises(ValueError, match="sphere_points"):
            ObservationConfig(sphere_points=bad)


def test_custom_points_pass_through():
    rng = np.random.default_rng(3)
    pts = rng.normal(size=(10, 3))
    points, angles = build_observation_points(FRAME, ObservationConfig(
        planes=["horizontal"], custom_points={"horizontal": pts}, angle_count=10))
    assert points.shape == (1, 10, 3) and len(angles) == 10
    np.testing.assert_allclose(points[0], pts)
    h, v = rng.normal(size=(7, 3)), rng.normal(size=(7, 3))
    points, angles = build_observation_points(FRAME, ObservationConfig(
        planes=["horizontal", "vertical"], custom_points={"horizontal": h, "vertical": v}, angle_count=7))
    assert points.shape == (2, 7, 3) and len(angles) == 7
    # a count that differs from angle_count: the angles follow the points, over the configured range
    cfg = ObservationConfig(planes=["horizontal"], custom_points={"horizontal": rng.normal(size=(15, 3))},
                            angle_count=37)
    points, angles = build_observation_points(FRAME, cfg)
    assert points.shape == (1, 15, 3) and len(angles) == 15
    assert angles[0] == cfg.angle_min_deg and angles[-1] == cfg.angle_max_deg


@pytest.mark.parametrize(("planes", "custom", "match"), [
    (["horizontal", "vertical"], {"horizontal": np.zeros((5, 3))}, "custom_points missing plane 'vertical'"),
    (["horizontal"], {"horizontal": np.zeros(15)}, r"must be \(N, 3\)"),
    (["horizontal"], {"horizontal": np.zeros((10, 2))}, r"must be \(N, 3\)"),
    (["horizontal", "vertical"], {"horizontal": np.zeros((10, 3)), "vertical": np.zeros((8, 3))},
     "same number of points"),
])
def test_custom_points_validation(planes, custom, match):
    with pytest.raises(ValueError, match=match):
        build_observation_points(FRAME, ObservationConfig(planes=planes, custom_points=custom))


def test_polar_arcs():
    points, angles = build_observation_points(FRAME, ObservationConfig(
        planes=["horizontal"], angle_min_deg=0.0, angle_max_deg=180.0, angle_count=3, distance_m=1.0))
    np.testing.assert_allclose(points[0, 0], FRAME.origin + FRAME.axis, atol=1e-12)   # 0 deg on the axis
    np.testing.assert_allclose(points[0, 2], FRAME.origin - FRAME.axis, atol=1e-12)   # 180 deg behind
    np.testing.assert_allclose(np.linalg.norm(points[0] - FRAME.origin, axis=1), 1.0)
    points, angles = build_observation_points(FRAME, ObservationConfig(planes=["vertical"], angle_count=91))
    assert points.shape == (1, 91, 3) and len(angles) == 91
    with pytest.raises(ValueError, match="Unknown plane"):
        build_observation_points(FRAME, ObservationConfig(planes=["foobar"]))
