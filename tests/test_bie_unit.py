"""Source-face multipliers and DP0 Neumann coefficients on tiny hand-made grids (host only): the
cases the reference's unit tests pin (tests/test_bie_unit.py:27-410, 420-830) -- axial projection,
the None fallbacks that keep the uniform-normal path bit-identical, the two-sided axial dipole,
radial tapers and bands, per-face and callable weights, and tag-average pressure."""
from __future__ import annotations

from types import SimpleNamespace

import numpy as np
import pytest

from hornlab_metal_bem_b200.bie import build_driver_neumann, build_source_face_scale, tag_average_pressure
from hornlab_metal_bem_b200.config import (
    AnnularProfile,
    CallableProfile,
    PerFaceProfile,
    SolveConfig,
    SourceMotion,
    TaperProfile,
    VelocityMode,
)

AXIS = np.array([0.0, 0.0, 1.0])
CENTER = np.zeros(3)


def _cap(theta: float):
    """Two unit-area-pair triangles with outward normals at +/- theta from +z (area-weighted mean +z)."""
    c, s = np.cos(theta), np.sin(theta)
    v = np.array([[0, 0, 0], [0, 1, 0], [-c, 0, s], [0, 0, 0], [0, 1, 0], [-c, 0, -s]], dtype=np.float64)
    return SimpleNamespace(vertices=v.T, elements=np.array([[0, 1, 2], [3, 4, 5]]).T)


def _radial(radii):
    """Small flat +z triangles with centroids on the x axis at the given radii."""
    e = 0.01
    v, f = [], []
    for r in radii:
        b = len(v)
        v += [[r - e, -e, 0.0], [r + e, -e, 0.0], [r, 2 * e, 0.0]]
        f.append([b, b + 1, b + 2])
    return SimpleNamespace(vertices=np.asarray(v).T, elements=np.asarray(f).T)


def _two_sided():
    """Equal-area faces, one facing +z and one facing -z (a thin diaphragm)."""
    v = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, -0.01], [0, 1, -0.01], [1, 0, -0.01]], dtype=np.float64)
    return SimpleNamespace(vertices=v.T, elements=np.array([[0, 1, 2], [3, 4, 5]]).T)


def _axial(**kw):
    return SolveConfig(velocity_sources={2: 1.0}, source_motion=SourceMotion.AXIAL, **kw)


def test_axial_projection():
    tags = np.array([2, 2])
    np.testing.assert_allclose(build_source_face_scale(_cap(0.0), tags, _axial(), AXIS, CENTER), [1, 1], atol=1e-12)
    th = np.deg2rad(35.0)
    np.testing.assert_allclose(build_source_face_scale(_cap(th), tags, _axial(), AXIS, CENTER),
                               [np.cos(th)] * 2, rtol=1e-9)
    th = np.deg2rad(40.0)
    s = build_source_face_scale(_cap(th), np.array([2, 7]), _axial(), AXIS, CENTER)
    np.testing.assert_allclose(s[0], np.cos(th), rtol=1e-9)
    assert s[1] == 0.0


def test_fallbacks_to_the_uniform_normal_path():
    tags = np.array([2, 2])
    grid = _cap(np.deg2rad(20.0))
    # no source face, a zero axis, or plain normal motion: None, so the scalar path stays bit-identical
    assert build_source_face_scale(grid, tags, SolveConfig(velocity_sources={99: 1.0},
                                                           source_motion=SourceMotion.AXIAL), AXIS, CENTER) is None
    assert build_source_face_scale(grid, tags, _axial(), np.zeros(3), CENTER) is None
    cfg = SolveConfig(velocity_sources={2: 1.0})
    assert build_source_face_scale(grid, tags, cfg, AXIS, CENTER) is None
    omega = 2 * np.pi * 1000.0
    direct = build_driver_neumann(2, tags, omega, cfg, np.complex64)
    via = build_driver_neumann(2, tags, omega, cfg, np.complex64, source_face_scale=None)
    assert np.array_equal(direct, via)


def test_two_sided_axial_tag_drives_a_dipole():
    tags = np.array([2, 2])
    cfg = _axial(velocity_mode=VelocityMode.VELOCITY)
    scale = build_source_face_scale(_two_sided(), tags, cfg, AXIS, CENTER)
    np.testing.assert_allclose(scale, [1.0, -1.0], atol=1e-12)
    q = build_driver_neumann(2, tags, 2 * np.pi * 1000.0, cfg, np.complex128, source_face_scale=scale)
    np.testing.assert_allclose(q[0], -q[1], rtol=1e-12)


def test_radial_profiles():
    tags3 = np.array([2, 2, 2])
    cfg = SolveConfig(velocity_sources={2: 1.0}, source_velocity_profiles={2: TaperProfile(start=0.0)})
    s = build_source_face_scale(_radial([0.0, 0.5, 1.0]), tags3, cfg, AXIS, CENTER)
    np.testing.assert_allclose(s, [1.0, 0.5, 0.0], atol=1e-12)     # raised cosine over the normalised radius
    cfg = SolveConfig(velocity_sources={2: 1.0}, source_velocity_profiles={2: AnnularProfile(0.4, 0.7)})
    np.testing.assert_allclose(build_source_face_scale(_radial([0.1, 0.5, 0.9]), tags3, cfg, AXIS, CENTER),
                               [0.0, 1.0, 0.0], atol=1e-12)


def test_per_face_and_callable_weights():
    tags = np.array([2, 2])
    w = np.array([1.0 + 0.5j, 0.25 - 0.25j])
    cfg = SolveConfig(velocity_sources={2: 1.0}, source_velocity_profiles={2: PerFaceProfile(w)})
    np.testing.assert_allclose(build_source_face_scale(_radial([0.0, 1.0]), tags, cfg, AXIS, CENTER), w, rtol=1e-12)
    seen = {}

    def cb(centroids, normals, axis, center):
        seen.update(centroids=centroids, normals=normals, axis=axis, center=center)
        return np.array([0.75 + 0.25j, 0.25 + 0.0j])

    cfg = SolveConfig(velocity_sources={2: 1.0}, source_velocity_profiles={2: CallableProfile(cb)})
    np.testing.assert_allclose(build_source_face_scale(_radial([0.0, 1.0]), tags, cfg, AXIS, CENTER),
                               [0.75 + 0.25j, 0.25 + 0.0j])
    assert seen["centroids"].shape == (2, 3)
    np.testing.assert_allclose(seen["normals"], [[0.0, 0.0, 1.0]] * 2)
    np.testing.assert_allclose(seen["axis"], AXIS)
    np.testing.assert_allclose(seen["center"], CENTER)
    bad = SolveConfig(velocity_sources={2: 1.0}, source_velocity_profiles={2: PerFaceProfile(np.ones(3))})
    with pytest.raises(ValueError, match="PerFaceProfile.weights"):
        build_source_face_scale(_radial([0.0, 1.0]), tags, bad, AXIS, CENTER)


def test_neumann_coefficients():
    tags = np.array([2, 2, 1])
    omega = 2 * np.pi * 1500.0
    vel = SolveConfig(velocity_sources={2: 1.0}, velocity_mode=VelocityMode.VELOCITY, air_density=1.205)
    q = build_driver_neumann(3, tags, omega, vel, np.complex128)
    np.testing.assert_allclose(q, [1j * 1.205 * omega] * 2 + [0.0])
    acc = SolveConfig(velocity_sources={2: 1.0}, velocity_mode=VelocityMode.ACCELERATION)
    q = build_driver_neumann(3, tags, omega, acc, np.complex128)
    np.testing.assert_allclose(q, [acc.air_density] * 2 + [0.0])     # i rho omega * (1 / (i omega))
    assert np.all(build_driver_neumann(3, tags, 0.0, acc, np.complex128) == 0)
    # a tag with an impedance (Robin) boundary is not driven
    rob = SolveConfig(velocity_sources={2: 1.0, 1: 0.5}, impedance_sources={1: 0.3 + 0.1j})
    q = build_driver_neumann(3, tags, omega, rob, np.complex128)
    assert q[2] == 0 and q[0] != 0
    # per-face axial scale multiplies the velocity face by face
    q = build_driver_neumann(3, tags, omega, vel, np.complex128, source_face_scale=np.array([1.0, 0.5, 0.0]))
    np.testing.assert_allclose(q[:2], 1j * 1.205 * omega * np.array([1.0, 0.5]))


def test_tag_average_pressure_is_area_weighted():
    areas = np.array([1.0, 3.0, 2.0])
    l2g = np.array([[0, 1, 2], [1, 2, 3], [3, 4, 5]])
    tags = np.array([2, 2, 1])
    p = np.array([1.0, 2.0, 3.0, 4.0, 5.0, 6.0], dtype=np.complex128)
    # face means 2 and 3, weights 1 and 3 -> (2 + 9) / 4
    assert tag_average_pressure(areas, l2g, tags, p, 2) == pytest.approx(11.0 / 4.0)
    assert tag_average_pressure(areas, l2g, tags, p, 1) == pytest.approx(5.0)
    assert tag_average_pressure(areas, l2g, tags, p, 9) == 0
