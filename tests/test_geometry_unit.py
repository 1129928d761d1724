"""Geometry buffers and the coupled-baffle aperture contract on hand-made grids (host only): the
rejections and the near-zero coordinate snap the reference's unit tests pin
(tests/test_metal_geometry.py:57-306); buffer contents on real meshes are golden-tested in
tests/test_frontend_golden.py."""
from __future__ import annotations

from types import SimpleNamespace

import numpy as np
import pytest

from hornlab_metal_bem_b200.geometry import (
    GeometryError,
    build_geometry_buffers,
    validate_native_infinite_baffle_aperture,
)

V4 = np.array([[0.0, 1.0, 0.0, 0.0], [0.0, 0.0, 1.0, 0.0], [0.0, 0.0, 0.0, 1.0]])
T2 = np.array([[0, 0], [1, 2], [2, 3]])


def _grid(v=V4, t=T2):
    return SimpleNamespace(vertices=v, elements=t, number_of_elements=t.shape[1])


def _p1(l2g=None, n=4):
    return SimpleNamespace(local2global=np.array([[0, 1, 2], [0, 2, 3]]) if l2g is None else l2g,
                           global_dof_count=n)


def _dp0(n=2):
    return SimpleNamespace(global_dof_count=n)


def test_tag_column_vector_is_accepted():
    b = build_geometry_buffers(_grid(), np.array([[1], [2]], dtype=np.int32), _p1())
    np.testing.assert_array_equal(b.physical_tags_i32, [1, 2])
    assert b.physical_tags_i32.dtype == np.int32


@pytest.mark.parametrize(("grid", "tags", "p1", "dp0", "match"), [
    (_grid(t=np.array([[1, 1], [2, 3], [3, 4]])), [1, 2], _p1(), None, "zero-based"),
    (_grid(), [1, 2], _p1(np.array([[0, 1, 2]])), None, "local2global"),
    (_grid(), [1, 2], _p1(np.array([[1, 2, 3], [1, 3, 4]])), None, "zero-based"),
    (_grid(), [1], _p1(), None, "physical_tags"),
    (_grid(t=np.array([[0], [1], [np.iinfo(np.int32).max + 1]], dtype=np.int64)), [1], _p1(np.array([[0, 1, 2]])),
     None, "int32"),
    (_grid(np.array([[0.0, 1.0, 2.0], [0.0, 0.0, 0.0], [0.0, 0.0, 0.0]]), np.array([[0], [1], [2]])), [1],
     _p1(np.array([[0, 1, 2]]), 3), _dp0(1), "zero area"),
    (_grid(), [1, 2], _p1(), _dp0(3), "dp0_space"),
])
def test_rejections(grid, tags, p1, dp0, match):
    with pytest.raises(GeometryError, match=match):
        build_geometry_buffers(grid, np.asarray(tags, dtype=np.int32), p1, dp0)
    assert issubclass(GeometryError, ValueError)


def test_near_zero_coordinates_snap_to_the_planes():
    v = np.array([[0.0, 1.0, 0.0, 0.0], [0.0, 0.0, 1.0, -5.0e-7], [5.0e-7, 2.0e-6, 0.0, 1.0]])
    b = build_geometry_buffers(_grid(v), np.array([1, 2], dtype=np.int32), _p1(), _dp0())
    assert b.vertices_3xn_f32[2, 0] == 0.0 and b.vertices_3xn_f32[1, 3] == 0.0
    assert b.vertices_3xn_f32[2, 1] == np.float32(2.0e-6)      # beyond the tolerance: kept
    assert v[2, 0] == 5.0e-7                                   # the caller's array is untouched


def _aperture(*, tag=7, z=0.0, flipped=False):
    v = np.array([[0.0, 1.0, 0.0], [0.0, 0.0, 1.0], [z, z, z]])
    t, l2g = (np.array([[0], [2], [1]]), np.array([[0, 2, 1]])) if flipped else \
        (np.array([[0], [1], [2]]), np.array([[0, 1, 2]]))
    return build_geometry_buffers(_grid(v, t), np.array([tag], dtype=np.int32), _p1(l2g, 3), _dp0(1))


def test_aperture_contract():
    good = _aperture(flipped=True)      # z = 0 disc with its normal -Z
    assert validate_native_infinite_baffle_aperture(good, 7) == 7
    assert validate_native_infinite_baffle_aperture(good, 7, symmetry_plane="yz+xz") == 7
    with pytest.raises(GeometryError, match="not present"):
        validate_native_infinite_baffle_aperture(_aperture(), 8)
    with pytest.raises(GeometryError, match="velocity_sources"):
        validate_native_infinite_baffle_aperture(_aperture(), 7, velocity_source_tags=[7])
    with pytest.raises(GeometryError, match="native_symmetry_plane='xy'"):
        validate_native_infinite_baffle_aperture(_aperture(), 7, symmetry_plane="xy")
    with pytest.raises(GeometryError, match="coplanar at Z=0"):
        validate_native_infinite_baffle_aperture(_aperture(z=1.0e-4, flipped=True), 7)
    with pytest.raises(GeometryError, match="normals pointing -Z"):
        validate_native_infinite_baffle_aperture(_aperture(), 7)
