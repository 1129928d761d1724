"""Front-end functions of the hot path against golden vectors from the reference's Python.

Fixtures: tests/golden/*.npz, written by tests/golden/make_golden.py from the
reference's own hornlab_metal_bem package (geometry buffers, frames,
observation arcs, Neumann rows, directivity, tag reductions).
"""
from __future__ import annotations

import numpy as np
import pytest
from types import SimpleNamespace

from conftest import golden, golden_buffers, grid_from_buffers, known_answers

from hornlab_metal_bem_b200 import generators as G
from hornlab_metal_bem_b200.bie import build_source_face_scale, compute_surface_pressure_avg, tag_average_pressure
from hornlab_metal_bem_b200.config import (
    AnnularProfile, ObservationConfig, PerFaceProfile, SolveConfig, TaperProfile,
)
from hornlab_metal_bem_b200.geometry import (
    GeometryError, build_geometry_buffers, validate_native_infinite_baffle_aperture, validate_native_symmetry_plane,
)
from hornlab_metal_bem_b200.mesh import make_pure_function_spaces
from hornlab_metal_bem_b200.observation import build_observation_points, infer_frame
from hornlab_metal_bem_b200.sweep import directivity_from_pressure, k_values, neumann_rows

GENERATED = ["ico2", "horn_quarter", "horn_full"]


def _generated_mesh(name):
    return {
        "ico2": lambda: G.icosphere(2, 0.1),
        "horn_quarter": lambda: G.horn(G.HornSpec(edge=0.014), quarter=True),
        "horn_full": lambda: G.horn(G.HornSpec(edge=0.016, flare=30.0, lip=0.004), quarter=False),
    }[name]()


@pytest.mark.parametrize("name", GENERATED)
def test_generated_meshes_are_reproducible(name):
    g = golden("geometry.npz")
    m = _generated_mesh(name)
    np.testing.assert_array_equal(np.asarray(m.grid.vertices), g[f"{name}__in_vertices"])
    np.testing.assert_array_equal(np.asarray(m.grid.elements), g[f"{name}__in_elements"])
    np.testing.assert_array_equal(np.asarray(m.physical_tags), g[f"{name}__in_tags"])


@pytest.mark.parametrize("name", GENERATED)
def test_geometry_buffers_match_reference(name):
    g = golden("geometry.npz")
    m = _generated_mesh(name)
    p1, dp0 = make_pure_function_spaces(m.grid)
    b = build_geometry_buffers(m.grid, m.physical_tags, p1, dp0)
    np.testing.assert_array_equal(b.vertices_3xn_f32, g[f"{name}__vertices"])
    np.testing.assert_array_equal(b.triangles_3xm_i32, g[f"{name}__triangles"])
    np.testing.assert_array_equal(b.p1_local2global_i32, g[f"{name}__l2g"])
    np.testing.assert_array_equal(b.physical_tags_i32, g[f"{name}__tags"])
    np.testing.assert_array_equal(b.triangle_areas_f32, g[f"{name}__areas"])
    np.testing.assert_array_equal(b.triangle_normals_3xm_f32, g[f"{name}__normals"])


@pytest.mark.parametrize("name", ["tiny", "near", "ib_box", "yzxz_quarter", "yzxz_full", "yz_half", "xy_full"])
def test_geometry_buffers_rebuild_reference_fixtures(name):
    ref = golden_buffers(name)
    grid = grid_from_buffers(ref)
    p1 = SimpleNamespace(local2global=ref.p1_local2global_i32, global_dof_count=ref.p1_dof_count)
    b = build_geometry_buffers(grid, ref.physical_tags_i32, p1)
    np.testing.assert_array_equal(b.triangle_areas_f32, ref.triangle_areas_f32)
    np.testing.assert_array_equal(b.triangle_normals_3xm_f32, ref.triangle_normals_3xm_f32)


def test_symmetry_and_aperture_validation_verdicts():
    verdicts = known_answers()["validation_verdicts"]
    for key, want in verdicts.items():
        parts = key.split("|")
        if parts[0] == "aperture":
            _, name, tag, plane = parts
            fn = lambda: validate_native_infinite_baffle_aperture(  # noqa: E731
                golden_buffers(name), int(tag), symmetry_plane=None if plane == "None" else plane)
        else:
            name, plane, chk = parts
            fn = lambda: validate_native_symmetry_plane(golden_buffers(name), plane, check_open_edges=chk == "True")  # noqa: E731
        if want == "ok":
            fn()
        else:
            with pytest.raises(GeometryError):
                fn()


def test_frames_and_observation_points_match_reference():
    fr = golden("frames.npz")
    cases = known_answers()["frame_cases"]
    for i, (name, tag, origin, plane) in enumerate(cases):
        m = _generated_mesh(name)
        f = infer_frame(m.grid, m.physical_tags, source_tag=tag, origin_at=origin, symmetry_plane=plane)
        for key in ("axis", "origin", "u", "v", "mouth_center", "source_center"):
            np.testing.assert_allclose(getattr(f, key), fr[f"{i}__{key}"], rtol=0, atol=1e-12, err_msg=f"{i} {key}")
        oc = ObservationConfig(planes=["horizontal", "vertical", "diagonal"], distance_m=2.0, angle_count=37)
        pts, ang = build_observation_points(f, oc)
        np.testing.assert_allclose(pts, fr[f"{i}__points"], rtol=0, atol=1e-12)
        np.testing.assert_allclose(ang, fr[f"{i}__angles"], rtol=0, atol=0)


def test_neumann_rows_match_reference():
    nm = golden("neumann.npz")
    m = _generated_mesh("horn_full")
    frame = infer_frame(m.grid, m.physical_tags, source_tag=2)
    perface = nm["perface"]
    cases = {
        "vel_normal": dict(velocity_mode="velocity"),
        "acc_normal": dict(velocity_mode="acceleration"),
        "vel_axial": dict(velocity_mode="velocity", source_motion="axial"),
        "acc_taper": dict(velocity_mode="acceleration", source_velocity_profiles={2: TaperProfile("raised_cosine", 0.5)}),
        "vel_taper_lin": dict(velocity_mode="velocity", source_velocity_profiles={2: TaperProfile("linear", 0.3)}),
        "vel_annular": dict(velocity_mode="velocity", source_velocity_profiles={2: AnnularProfile(0.2, 0.8)}),
        "vel_perface": dict(velocity_mode="velocity", source_velocity_profiles={2: PerFaceProfile(perface)}),
        "vel_two_tags": dict(velocity_mode="velocity", velocity_sources={2: 1.0, 1: 0.25}, air_density=1.205),
        "robin_skip": dict(velocity_mode="velocity", velocity_sources={2: 1.0, 1: 0.5}, impedance_sources={1: 0.3 + 0.1j}),
    }
    assert sorted(cases) == sorted(known_answers()["neumann_cases"])
    freqs = nm["freqs"]
    for name, kw in cases.items():
        cfg = SolveConfig(**kw)
        scale = build_source_face_scale(m.grid, m.physical_tags, cfg, frame.axis, frame.source_center)
        rows = neumann_rows(m.info.n_triangles, m.physical_tags, freqs, cfg, scale)
        np.testing.assert_allclose(rows, nm[f"{name}__rows"], rtol=1e-6, atol=1e-6, err_msg=name)
        k_re, _ = k_values(freqs, cfg)
        np.testing.assert_array_equal(k_re, nm[f"{name}__k"])


def test_directivity_and_reductions_match_reference():
    rd = golden("reductions.npz")
    p = rd["pressure"]
    for i in range(p.shape[0]):
        np.testing.assert_allclose(directivity_from_pressure(p[i], 0), rd["directivity"][i], rtol=0, atol=1e-12)
        np.testing.assert_allclose(directivity_from_pressure(p[i], 3), rd["directivity_idx3"][i], rtol=0, atol=1e-12)
    m = _generated_mesh("horn_full")
    p1, _ = make_pure_function_spaces(m.grid)
    ps = rd["surface"]
    imp = tag_average_pressure(m.grid.volumes, p1.local2global, m.physical_tags, ps, 2)
    assert abs(imp - complex(rd["impedance_tag2"])) < 1e-12
    pav = compute_surface_pressure_avg(m.grid.volumes, p1.local2global, m.physical_tags, ps, [1, 2, 9])
    np.testing.assert_allclose([pav[1], pav[2], pav[9]], rd["pavg"], rtol=0, atol=1e-12)
