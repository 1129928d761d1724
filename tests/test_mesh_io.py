"""Gmsh surface meshes and the ``load_mesh`` pipeline (host only).

The reference reads ``.msh`` files with meshio (hornlab_metal_bem/mesh.py:51-157), which is not installed
here; this package reads ASCII MSH 2.2 and 4.1 itself.  The steps after reading follow the reference:
seam-vertex merging on a ``merge_tol`` lattice (vertices in sorted key order when anything merges,
mesh.py:387-408), removal of triangles that merging made degenerate, the outward-winding check with
optional repair (mesh.py:411-443), the coupled-baffle contract (negative signed volume, aperture normals
-Z, mesh.py:454-506), the velocity-source group check (mesh.py:520+) and the reduced-mesh warning
(mesh.py:287-309).
"""
from __future__ import annotations

import warnings

import numpy as np
import pytest

from hornlab_metal_bem_b200 import generators as G
from hornlab_metal_bem_b200.mesh import MeshError, load_mesh, read_gmsh, signed_volume_indicator, write_gmsh22

# closed, outward-wound tetrahedron: three faces on the coordinate planes (tag 1), the slanted one (tag 2)
TET_V = np.array([[0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [0.0, 1.0, 0.0], [0.0, 0.0, 1.0]])
TET_F = np.array([[0, 2, 1], [0, 1, 3], [0, 3, 2], [1, 2, 3]])
TET_TAGS = np.array([1, 1, 1, 2])
NAMES = {1: "wall", 2: "throat"}


def _mesh_arrays(m):
    return m.grid.vertices.T, m.grid.elements.T, np.asarray(m.physical_tags)


def test_msh22_round_trip_keeps_geometry_tags_and_names(tmp_path):
    src = G.icosphere(1, 0.1)
    v, f, _ = _mesh_arrays(src)
    tags = np.where(v[f].mean(axis=1)[:, 2] > 0.05, 2, 1)
    path = tmp_path / "sphere.msh"
    write_gmsh22(path, v, f, tags, NAMES)
    m = load_mesh(path)
    v2, f2, t2 = _mesh_arrays(m)
    np.testing.assert_array_equal(v2, v)        # repr() floats round-trip exactly, nothing merges
    np.testing.assert_array_equal(f2, f)
    np.testing.assert_array_equal(t2, tags)
    assert m.info.physical_groups == NAMES
    assert m.info.n_vertices == v.shape[0] and m.info.n_triangles == f.shape[0]
    scaled = load_mesh(path, scale=1e3)
    np.testing.assert_allclose(scaled.grid.vertices.T, v * 1e3, rtol=1e-15)


def test_msh41_ascii_entities_give_physical_tags(tmp_path):
    lines = ["$MeshFormat", "4.1 0 8", "$EndMeshFormat",
             "$PhysicalNames", "2", '2 1 "wall"', '2 2 "throat"', "$EndPhysicalNames",
             "$Entities", "0 1 2 0",
             "1 0 0 0 1 0 0 0 0",                      # one curve, no physical tag
             "1 0 0 0 1 1 1 1 1 0",                    # surface 1 -> physical 1
             "2 0 0 0 1 1 1 1 2 0",                    # surface 2 -> physical 2
             "$EndEntities",
             "$Nodes", "1 4 1 4", "2 1 0 4", "1", "2", "3", "4"]
    lines += [f"{float(x)!r} {float(y)!r} {float(z)!r}" for x, y, z in TET_V]
    lines += ["$EndNodes", "$Elements", "3 5 1 5",
              "1 1 1 1", "1 1 2",                       # a line element: skipped
              "2 1 2 3"]
    lines += [f"{2 + i} {a + 1} {b + 1} {c + 1}" for i, (a, b, c) in enumerate(TET_F[:3])]
    lines += ["2 2 2 1", f"5 {TET_F[3, 0] + 1} {TET_F[3, 1] + 1} {TET_F[3, 2] + 1}", "$EndElements", ""]
    path = tmp_path / "tet41.msh"
    path.write_text("\n".join(lines))
    pts, tris, tags, names = read_gmsh(path)
    np.testing.assert_array_equal(pts, TET_V)
    np.testing.assert_array_equal(tris, TET_F)
    np.testing.assert_array_equal(tags, TET_TAGS)
    assert names == NAMES
    m = load_mesh(path)
    assert m.info.n_triangles == 4 and signed_volume_indicator(*_mesh_arrays(m)[:2]) > 0


def test_seam_vertices_merge_and_collapsed_triangles_drop(tmp_path):
    # triangle soup: every face with its own three nodes, plus one triangle that collapses when merged
    soup_v = TET_V[TET_F.reshape(-1)]
    soup_f = np.arange(12).reshape(4, 3)
    soup_v = np.vstack([soup_v, TET_V[0] + 2e-10])
    soup_f = np.vstack([soup_f, [[0, 12, 1]]])
    path = tmp_path / "soup.msh"
    write_gmsh22(path, soup_v, soup_f, np.append(TET_TAGS, 1), NAMES)
    m = load_mesh(path, merge_tol=1e-9)
    v, f, t = _mesh_arrays(m)
    # merged vertices in sorted lattice-key order: (0,0,0) (0,0,1) (0,1,0) (1,0,0)
    order = np.lexsort(TET_V.T[::-1])
    np.testing.assert_array_equal(v, TET_V[order])
    remap = np.empty(4, np.int64)
    remap[order] = np.arange(4)
    np.testing.assert_array_equal(f, remap[TET_F])
    np.testing.assert_array_equal(t, TET_TAGS)
    # without merging nothing collapses and the 13 soup nodes stay
    raw = load_mesh(path, merge_tol=0.0, validate=False)
    assert raw.info.n_vertices == 13 and raw.info.n_triangles == 5


def test_inward_winding_is_rejected_unless_repaired(tmp_path):
    path = tmp_path / "inward.msh"
    write_gmsh22(path, TET_V, TET_F[:, [0, 2, 1]], TET_TAGS, NAMES)
    with pytest.raises(MeshError, match="winding appears inward"):
        load_mesh(path)
    m = load_mesh(path, repair_normals=True)
    v, f, _ = _mesh_arrays(m)
    assert signed_volume_indicator(v, f) > 0
    np.testing.assert_array_equal(f, TET_F)
    load_mesh(path, validate=False)   # no checks, no repair


def test_group_check_needs_a_velocity_source(tmp_path):
    path = tmp_path / "rigid.msh"
    write_gmsh22(path, TET_V, TET_F, np.ones(4, int), {1: "wall"})
    with pytest.raises(MeshError, match="No velocity source"):
        load_mesh(path)


def test_coupled_baffle_contract(tmp_path):
    b = G.baffled_horn(G.HornSpec(edge=0.02))
    v, f, t = _mesh_arrays(b)
    path = tmp_path / "baffled.msh"
    write_gmsh22(path, v, f, t, b.info.physical_groups)
    m = load_mesh(path)       # aperture found by its group name; negative signed volume, normals -Z
    assert m.info.n_triangles == f.shape[0]
    flipped = tmp_path / "baffled_flipped.msh"
    write_gmsh22(flipped, v, f[:, [0, 2, 1]], t, b.info.physical_groups)
    with pytest.raises(MeshError, match="winding appears inverse"):
        load_mesh(flipped)


def test_reduced_mesh_warning(tmp_path):
    q = G.horn(G.HornSpec(edge=0.02), quarter=True)
    v, f, t = _mesh_arrays(q)
    path = tmp_path / "quarter.msh"
    write_gmsh22(path, v, f, t, {1: "wall", 2: "throat"})
    with pytest.warns(RuntimeWarning, match="'yz\\+xz'"):
        load_mesh(path)
    with warnings.catch_warnings():
        warnings.simplefilter("error")
        load_mesh(path, native_symmetry_plane="yz+xz")


def test_reader_errors(tmp_path):
    with pytest.raises(MeshError, match="not found"):
        load_mesh(tmp_path / "missing.msh")
    binary = tmp_path / "binary.msh"
    binary.write_text("$MeshFormat\n2.2 1 8\n$EndMeshFormat\n")
    with pytest.raises(MeshError, match="binary"):
        read_gmsh(binary)
    old = tmp_path / "v3.msh"
    old.write_text("$MeshFormat\n3.0 0 8\n$EndMeshFormat\n")
    with pytest.raises(MeshError, match="unsupported MSH version"):
        read_gmsh(old)
    lines_only = tmp_path / "lines.msh"
    lines_only.write_text("$MeshFormat\n2.2 0 8\n$EndMeshFormat\n$Nodes\n2\n1 0 0 0\n2 1 0 0\n$EndNodes\n"
                          "$Elements\n1\n1 1 2 1 1 1 2\n$EndElements\n")
    with pytest.raises(MeshError, match="No triangles"):
        read_gmsh(lines_only)
    not_msh = tmp_path / "x.msh"
    not_msh.write_text("solid x\nendsolid x\n")
    with pytest.raises(MeshError, match="not a Gmsh"):
        read_gmsh(not_msh)


def test_pure_grid_and_function_spaces():
    """Array-only grid and P1 / DP0 spaces (reference tests/test_pure_mesh.py:19-56)."""
    from hornlab_metal_bem_b200.mesh import make_pure_function_spaces, make_pure_grid

    g = make_pure_grid(TET_V, np.array([[0, 1, 2], [0, 1, 3]]))
    assert g.vertices.shape == (3, 4) and g.elements.shape == (3, 2) and g.number_of_elements == 2
    np.testing.assert_allclose(g.volumes, [0.5, 0.5])
    p1, dp0 = make_pure_function_spaces(make_pure_grid(np.eye(3), np.array([[0, 1, 2]])))
    np.testing.assert_array_equal(p1.local2global, [[0, 1, 2]])
    assert p1.global_dof_count == 3 and dp0.global_dof_count == 1


@pytest.mark.parametrize(("verts", "tris", "plane"), [
    ([[0, 0, 0], [0, 1, 0], [0, 0, 1], [1, 0.2, 0.3]], [[0, 1, 3], [0, 3, 2], [1, 2, 3]], "yz"),
    ([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], [[0, 1, 2], [1, 3, 2]], "yz+xz"),
    ([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0.2, 0.3, 1]], [[0, 1, 3], [0, 3, 2], [1, 2, 3]], "xy"),
    (TET_V, TET_F, None),     # closed: no open rim, no reduced plane
])
def test_reduced_symmetry_plane_detection(verts, tris, plane):
    """Open rims lying on the coordinate planes name the mirror plane(s) of a reduced mesh (reference
    tests/test_pure_mesh.py:97-160)."""
    from hornlab_metal_bem_b200.mesh import detect_reduced_symmetry_plane

    assert detect_reduced_symmetry_plane(np.asarray(verts, float), np.asarray(tris)) == plane
