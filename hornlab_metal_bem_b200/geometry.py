"""Validated geometry buffers handed to the CUDA session.

Restates ``hornlab_metal_bem/metal/geometry.py`` of the reference:

* ``build_geometry_buffers`` (``geometry.py:78-140``): vertices (3, V) f32 with
  ``|x| <= 1e-6`` snapped to 0 (so mirrored vertices match the 1e-6 lattice
  used for image-pair detection), triangles (3, T) i32, tags (T,), P1
  local2global (T, 3), areas (T,) and unit normals (3, T) computed in f64 and
  stored f32; zero-based, compact, in-range indices are enforced.
* ``validate_native_symmetry_plane`` (``geometry.py:143-213``) and
  ``validate_native_infinite_baffle_aperture`` (``geometry.py:216-306``).
"""
from __future__ import annotations

from dataclasses import dataclass
from numbers import Integral
from typing import Any

import numpy as np
from numpy.typing import NDArray

from .config import NATIVE_SYMMETRY_PLANES
from .mesh import open_boundary_edges

PLANE_SNAP_TOLERANCE = 1.0e-6


class GeometryError(ValueError):
    """Geometry or function-space metadata that cannot satisfy the session contract."""


# Drop-in alias for callers that catch the reference's exception type name.
MetalGeometryError = GeometryError


@dataclass(frozen=True)
class GeometryBuffers:
    vertices_3xn_f32: NDArray[np.float32]
    triangles_3xm_i32: NDArray[np.int32]
    physical_tags_i32: NDArray[np.int32]
    p1_local2global_i32: NDArray[np.int32]
    triangle_areas_f32: NDArray[np.float32]
    triangle_normals_3xm_f32: NDArray[np.float32]
    p1_dof_count: int
    dp0_dof_count: int

    @property
    def n_vertices(self) -> int:
        return int(self.vertices_3xn_f32.shape[1])

    @property
    def n_triangles(self) -> int:
        return int(self.triangles_3xm_i32.shape[1])

    @property
    def triangles_nx3_i32(self) -> NDArray[np.int32]:
        return np.ascontiguousarray(self.triangles_3xm_i32.T)


def _int_array(name: str, value) -> NDArray[np.int32]:
    arr = np.asarray(value)
    if not np.issubdtype(arr.dtype, np.integer):
        raise GeometryError(f"{name} must contain integer values")
    if arr.size == 0:
        raise GeometryError(f"{name} must not be empty")
    lo, hi = int(arr.min()), int(arr.max())
    info = np.iinfo(np.int32)
    if lo < info.min or hi > info.max:
        raise GeometryError(f"{name} values must fit int32, got range [{lo}, {hi}]")
    return np.asarray(arr, dtype=np.int32)


def _check_zero_based(name: str, idx, upper: int | None = None) -> None:
    lo, hi = int(idx.min()), int(idx.max())
    if lo < 0:
        raise GeometryError(f"{name} indices must be zero-based and nonnegative")
    if lo != 0:
        raise GeometryError(
            f"{name} indices must be compact zero-based arrays with minimum 0; got minimum {lo}"
        )
    if upper is not None and hi >= upper:
        raise GeometryError(f"{name} indices must be zero-based and less than {upper}; got max {hi}")


def _nonneg_int(name: str, value) -> int:
    if isinstance(value, bool):
        raise GeometryError(f"{name} must be an integer")
    try:
        out = int(value)
    except (TypeError, ValueError) as exc:
        raise GeometryError(f"{name} must be an integer") from exc
    if out < 0:
        raise GeometryError(f"{name} must be nonnegative")
    return out


def build_geometry_buffers(grid: Any, physical_tags: Any, p1_space: Any, dp0_space: Any | None = None) -> GeometryBuffers:
    if not hasattr(grid, "vertices"):
        raise GeometryError("grid must expose a vertices array")
    verts = np.asarray(grid.vertices)
    if verts.ndim != 2 or verts.shape[0] != 3:
        raise GeometryError(f"grid.vertices must have shape (3, n_vertices), got {verts.shape}")
    if verts.shape[1] == 0:
        raise GeometryError("grid.vertices must contain at least one vertex")
    verts = np.array(verts, dtype=np.float64)
    if not np.all(np.isfinite(verts)):
        raise GeometryError("grid.vertices must contain only finite values")
    verts[np.abs(verts) <= PLANE_SNAP_TOLERANCE] = 0.0

    if not hasattr(grid, "elements"):
        raise GeometryError("grid must expose an elements array")
    elems = np.asarray(grid.elements)
    if elems.ndim != 2 or elems.shape[0] != 3:
        raise GeometryError(f"grid.elements must have shape (3, n_triangles), got {elems.shape}")
    if elems.shape[1] == 0:
        raise GeometryError("grid.elements must contain at least one triangle")
    tris = _int_array("grid.elements", elems)
    _check_zero_based("grid.elements", tris, upper=verts.shape[1])
    rows = tris.T
    rep = (rows[:, 0] == rows[:, 1]) | (rows[:, 1] == rows[:, 2]) | (rows[:, 0] == rows[:, 2])
    if np.any(rep):
        raise GeometryError(f"grid.elements triangle {int(np.flatnonzero(rep)[0])} repeats a vertex index")
    n_tri = int(tris.shape[1])
    if hasattr(grid, "number_of_elements"):
        cnt = _nonneg_int("grid.number_of_elements", grid.number_of_elements)
        if cnt != n_tri:
            raise GeometryError(
                f"grid.number_of_elements={cnt} does not match elements shape with {n_tri} triangles"
            )

    tags = np.asarray(physical_tags)
    if tags.ndim == 2 and 1 in tags.shape:
        tags = tags.reshape(-1)
    if tags.ndim != 1:
        raise GeometryError(f"physical_tags must be a 1D array, got shape {tags.shape}")
    if tags.shape != (n_tri,):
        raise GeometryError(
            f"physical_tags must have one value per triangle: expected {(n_tri,)}, got {tags.shape}"
        )
    tags = np.ascontiguousarray(_int_array("physical_tags", tags))

    if not hasattr(p1_space, "local2global"):
        raise GeometryError("p1_space must expose a local2global array")
    l2g_raw = np.asarray(p1_space.local2global)
    if l2g_raw.shape != (n_tri, 3):
        raise GeometryError(
            f"p1_space.local2global must have shape (n_triangles, 3): expected {(n_tri, 3)}, got {l2g_raw.shape}"
        )
    l2g = _int_array("p1_space.local2global", l2g_raw)
    _check_zero_based("p1_space.local2global", l2g)
    need = int(l2g.max()) + 1
    p1_count = _nonneg_int("p1_space.global_dof_count", getattr(p1_space, "global_dof_count", need))
    if p1_count < need:
        raise GeometryError(
            f"p1_space.global_dof_count is smaller than local2global requires: {p1_count} < {need}"
        )
    if dp0_space is None:
        dp0_count = n_tri
    else:
        dp0_count = _nonneg_int("dp0_space.global_dof_count", getattr(dp0_space, "global_dof_count", n_tri))
        if dp0_count != n_tri:
            raise GeometryError(f"dp0_space.global_dof_count must equal n_triangles: {dp0_count} != {n_tri}")

    pts = verts.T
    p0, p1, p2 = pts[rows[:, 0]], pts[rows[:, 1]], pts[rows[:, 2]]
    cross = np.cross(p1 - p0, p2 - p0)
    twice = np.linalg.norm(cross, axis=1)
    if np.any(twice <= 0.0):
        raise GeometryError(f"grid.elements triangle {int(np.flatnonzero(twice <= 0.0)[0])} has zero area")
    normals = cross / twice[:, None]
    areas = 0.5 * twice
    if not (np.all(np.isfinite(normals)) and np.all(np.isfinite(areas))):
        raise GeometryError("triangle areas/normals must be finite")
    return GeometryBuffers(
        vertices_3xn_f32=np.ascontiguousarray(verts, dtype=np.float32),
        triangles_3xm_i32=np.ascontiguousarray(tris, dtype=np.int32),
        physical_tags_i32=tags,
        p1_local2global_i32=np.ascontiguousarray(l2g, dtype=np.int32),
        triangle_areas_f32=np.ascontiguousarray(areas, dtype=np.float32),
        triangle_normals_3xm_f32=np.ascontiguousarray(normals.T, dtype=np.float32),
        p1_dof_count=p1_count,
        dp0_dof_count=dp0_count,
    )


# Drop-in alias for the reference's builder name.
build_metal_geometry_buffers = build_geometry_buffers


def _plane_components(plane: str) -> list[tuple[int, str, str]]:
    comps = []
    if "yz" in plane:
        comps.append((0, "x", "X=0"))
    if "xz" in plane:
        comps.append((1, "y", "Y=0"))
    if plane == "xy":
        comps.append((2, "z", "Z=0"))
    return comps


def validate_native_symmetry_plane(
    buffers: GeometryBuffers,
    symmetry_plane: str | None,
    *,
    tolerance: float = 1.0e-7,
    check_open_edges: bool = True,
) -> str | None:
    """Positive-side reduced mesh, vertices on each image plane, no face lying on a plane."""
    if symmetry_plane is None:
        return None
    plane = str(symmetry_plane).strip().lower()
    if plane not in NATIVE_SYMMETRY_PLANES:
        raise GeometryError("native_symmetry_plane currently supports 'yz', 'xz', 'xy', and 'yz+xz'")
    coords = np.asarray(buffers.vertices_3xn_f32, dtype=np.float64)
    if coords.shape[1] == 0:
        raise GeometryError(f"native_symmetry_plane={plane!r} requires vertices")
    tris = buffers.triangles_nx3_i32
    used = np.unique(tris.reshape(-1))
    for comp, name, label in _plane_components(plane):
        vals = coords[comp]
        lo = float(np.min(vals[used]))
        if lo < -tolerance:
            raise GeometryError(
                f"native_symmetry_plane={plane!r} requires a positive-{name} reduced-domain mesh; "
                f"minimum {name.upper()} is {lo:.6g}"
            )
        if not np.any(np.abs(vals[used]) <= tolerance):
            raise GeometryError(f"native_symmetry_plane={plane!r} requires boundary vertices on {name.upper()}=0")
        flat = np.all(np.abs(vals[tris]) <= tolerance, axis=1)
        if np.any(flat):
            raise GeometryError(
                f"native_symmetry_plane={plane!r} treats {label} as an image plane, not a physical "
                f"boundary; triangle {int(np.flatnonzero(flat)[0])} lies entirely on the plane"
            )
    if check_open_edges:
        edges = open_boundary_edges(tris)
        if edges.size:
            comps = _plane_components(plane)
            ok = np.zeros(edges.shape[0], dtype=bool)
            for comp, _, _ in comps:
                ok |= np.all(np.abs(coords[comp, edges]) <= PLANE_SNAP_TOLERANCE, axis=1)
            if not np.all(ok):
                first = int(np.flatnonzero(~ok)[0])
                edge = tuple(int(v) for v in edges[first])
                labels = " or ".join(c[2] for c in comps)
                raise GeometryError(
                    f"native_symmetry_plane={plane!r} requires every open boundary edge to lie on "
                    f"{labels}; boundary edge {first} with vertices {edge} is off the requested "
                    "symmetry plane(s). If this rim is a real free edge of the full (reduced + "
                    "mirrored) geometry (e.g. an open horn mouth), set "
                    "SolveConfig.native_check_open_edges=False."
                )
    return plane


def validate_native_infinite_baffle_aperture(
    buffers: GeometryBuffers,
    aperture_tag: int | None,
    *,
    velocity_source_tags=None,
    symmetry_plane: str | None = None,
    tolerance: float = 1.0e-6,
) -> int | None:
    """Aperture faces coplanar at z = 0 with normals -Z; tag distinct from the driven tags."""
    if aperture_tag is None:
        return None
    if isinstance(aperture_tag, bool) or not isinstance(aperture_tag, Integral) or int(aperture_tag) <= 0:
        raise GeometryError("aperture_tag must be a positive int or None")
    tag = int(aperture_tag)
    plane = None if symmetry_plane is None else str(symmetry_plane).strip().lower()
    if plane == "xy":
        raise GeometryError(
            "aperture_tag coupled infinite-baffle mode does not compose with "
            "native_symmetry_plane='xy'; use None, 'yz', 'xz', or 'yz+xz'"
        )
    if plane is not None and plane not in ("yz", "xz", "yz+xz"):
        raise GeometryError(
            "aperture_tag coupled infinite-baffle mode requires native_symmetry_plane to be None, "
            "'yz', 'xz', or 'yz+xz'"
        )
    sources: set[int] = set()
    for t in velocity_source_tags or ():
        if isinstance(t, bool) or not isinstance(t, Integral) or int(t) <= 0:
            raise GeometryError("velocity_source_tags must be positive ints")
        sources.add(int(t))
    if tag in sources:
        raise GeometryError("aperture_tag must not also be listed in velocity_sources")
    tags = np.asarray(buffers.physical_tags_i32)
    mask = tags == tag
    if not np.any(mask):
        raise GeometryError(
            f"aperture_tag {tag} is not present in the mesh; available physical tags: "
            f"{sorted(int(v) for v in np.unique(tags))}"
        )
    coords = np.asarray(buffers.vertices_3xn_f32, dtype=np.float64)
    zmax = float(np.max(np.abs(coords[2, buffers.triangles_nx3_i32[mask]])))
    if zmax > tolerance:
        raise GeometryError(f"aperture_tag triangles must be coplanar at Z=0; max |Z| is {zmax:.6g}")
    nrm = np.asarray(buffers.triangle_normals_3xm_f32, dtype=np.float64)[:, mask]
    ntol = max(float(tolerance), 1.0e-5)
    bad = (np.hypot(nrm[0], nrm[1]) > ntol) | (nrm[2] > -1.0 + ntol) | (nrm[2] >= 0.0)
    if np.any(bad):
        j = int(np.flatnonzero(bad)[0])
        first = int(np.flatnonzero(mask)[j])
        raise GeometryError(
            f"aperture_tag triangles must have normals pointing -Z; triangle {first} normal is "
            f"({nrm[0, j]:.6g}, {nrm[1, j]:.6g}, {nrm[2, j]:.6g})"
        )
    return tag
