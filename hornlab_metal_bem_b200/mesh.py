"""Surface-mesh loading, P1/DP0 function spaces and mesh checks.

Behaviour follows ``hornlab_metal_bem/mesh.py`` of the reference:

* ``load_mesh`` (``mesh.py:51-157``): read triangles + physical tags, merge
  coincident seam vertices, drop degenerate triangles, check outward winding
  by the signed-volume indicator, check the coupled infinite-baffle aperture
  contract, warn when a mesh looks mirror-reduced but no symmetry plane is set.
* ``make_pure_grid`` / ``make_pure_function_spaces`` (``mesh.py:160-197``):
  P1 = one dof per vertex, DP0 = one dof per triangle.

The reference reads ``.msh`` files through meshio, which this image does not
ship, so the Gmsh reader here is self-contained: MSH 2.2 and 4.1 ASCII, taking
a triangle's physical tag from its element tags (2.2) or its surface entity
(4.1) exactly as meshio's ``gmsh:physical`` cell data does.
"""
from __future__ import annotations

import logging
import warnings
from dataclasses import dataclass
from numbers import Integral
from pathlib import Path

import numpy as np
from numpy.typing import NDArray

from .result import MeshInfo

logger = logging.getLogger(__name__)

SYMMETRY_SNAP_TOLERANCE = 1.0e-6
CANONICAL_APERTURE_TAG = 12
CANONICAL_APERTURE_NAME = "mouth_aperture"


class MeshError(Exception):
    pass


@dataclass
class LoadedMesh:
    grid: object
    physical_tags: NDArray[np.int32]
    info: MeshInfo


@dataclass(frozen=True)
class PureGrid:
    """Array-only grid: ``vertices`` (3, V) f64, ``elements`` (3, T) i32, ``volumes`` (T,) areas."""

    vertices: NDArray[np.float64]
    elements: NDArray[np.int32]
    volumes: NDArray[np.float64]

    @property
    def number_of_elements(self) -> int:
        return int(self.elements.shape[1])


@dataclass(frozen=True)
class PureFunctionSpace:
    local2global: NDArray[np.int32]
    global_dof_count: int


# --------------------------------------------------------------------------- #
# Gmsh ASCII reader
# --------------------------------------------------------------------------- #
def _sections(text: str) -> dict[str, list[str]]:
    out: dict[str, list[str]] = {}
    lines = text.splitlines()
    i = 0
    while i < len(lines):
        line = lines[i].strip()
        if line.startswith("$") and not line.startswith("$End"):
            name = line[1:]
            body: list[str] = []
            i += 1
            while i < len(lines) and lines[i].strip() != f"$End{name}":
                body.append(lines[i])
                i += 1
            out.setdefault(name, body)
        i += 1
    return out


def _physical_names(body: list[str] | None) -> dict[int, str]:
    names: dict[int, str] = {}
    for raw in (body or [])[1:]:
        parts = raw.strip().split(maxsplit=2)
        if len(parts) < 3 or not parts[0].isdigit():
            continue
        if int(parts[0]) == 2:
            names[int(parts[1])] = parts[2].strip().strip('"')
    return names


def _read_msh22(sec: dict[str, list[str]]):
    node_lines = sec["Nodes"]
    count = int(node_lines[0])
    ids = np.empty(count, dtype=np.int64)
    pts = np.empty((count, 3), dtype=np.float64)
    for n, raw in enumerate(node_lines[1 : count + 1]):
        f = raw.split()
        ids[n] = int(f[0])
        pts[n] = (float(f[1]), float(f[2]), float(f[3]))
    index = {int(t): n for n, t in enumerate(ids)}
    tris: list[tuple[int, int, int]] = []
    tags: list[int] = []
    elem_lines = sec["Elements"]
    for raw in elem_lines[1 : int(elem_lines[0]) + 1]:
        f = [int(v) for v in raw.split()]
        if f[1] != 2:
            continue
        ntags = f[2]
        phys = f[3] if ntags > 0 else 0
        nodes = f[3 + ntags : 6 + ntags]
        tris.append(tuple(index[v] for v in nodes))
        tags.append(phys)
    return pts, np.asarray(tris, dtype=np.int64).reshape(-1, 3), np.asarray(tags, dtype=np.int32)


def _read_msh41(sec: dict[str, list[str]]):
    surface_phys: dict[int, int] = {}
    ent = sec.get("Entities")
    if ent:
        head = [int(v) for v in ent[0].split()]
        n_pts, n_curves, n_surf = head[0], head[1], head[2]
        for raw in ent[1 + n_pts + n_curves : 1 + n_pts + n_curves + n_surf]:
            f = raw.split()
            tag = int(f[0])
            nphys = int(f[7])
            surface_phys[tag] = int(f[8]) if nphys > 0 else 0
    node_lines = sec["Nodes"]
    head = [int(v) for v in node_lines[0].split()]
    n_blocks, n_nodes = head[0], head[1]
    ids = np.empty(n_nodes, dtype=np.int64)
    pts = np.empty((n_nodes, 3), dtype=np.float64)
    cursor, filled = 1, 0
    for _ in range(n_blocks):
        f = node_lines[cursor].split()
        nblock = int(f[3])
        parametric = int(f[2])
        if parametric:
            raise MeshError("parametric MSH 4.1 nodes are not supported")
        cursor += 1
        for j in range(nblock):
            ids[filled + j] = int(node_lines[cursor + j])
        cursor += nblock
        for j in range(nblock):
            c = node_lines[cursor + j].split()
            pts[filled + j] = (float(c[0]), float(c[1]), float(c[2]))
        cursor += nblock
        filled += nblock
    index = {int(t): n for n, t in enumerate(ids)}
    elem_lines = sec["Elements"]
    head = [int(v) for v in elem_lines[0].split()]
    cursor = 1
    tris: list[tuple[int, int, int]] = []
    tags: list[int] = []
    for _ in range(head[0]):
        f = [int(v) for v in elem_lines[cursor].split()]
        dim, entity, etype, nblock = f
        cursor += 1
        if etype == 2 and dim == 2:
            phys = surface_phys.get(entity, 0)
            for raw in elem_lines[cursor : cursor + nblock]:
                e = [int(v) for v in raw.split()]
                tris.append((index[e[1]], index[e[2]], index[e[3]]))
                tags.append(phys)
        cursor += nblock
    return pts, np.asarray(tris, dtype=np.int64).reshape(-1, 3), np.asarray(tags, dtype=np.int32)


def read_gmsh(path: str | Path):
    """Return ``(points (V,3) f64, triangles (T,3) i32, tags (T,) i32, names)``."""
    text = Path(path).read_text(encoding="utf-8", errors="replace")
    sec = _sections(text)
    if "MeshFormat" not in sec:
        raise MeshError(f"{path} is not a Gmsh .msh file")
    fmt = sec["MeshFormat"][0].split()
    version, filetype = fmt[0], int(fmt[1])
    if filetype != 0:
        raise MeshError("binary .msh files are not supported; export ASCII")
    if version.startswith("2"):
        pts, tris, tags = _read_msh22(sec)
    elif version.startswith("4"):
        pts, tris, tags = _read_msh41(sec)
    else:
        raise MeshError(f"unsupported MSH version {version}")
    if tris.shape[0] == 0:
        raise MeshError("No triangles found in mesh")
    return pts, tris.astype(np.int32), tags, _physical_names(sec.get("PhysicalNames"))


def write_gmsh22(path: str | Path, points, triangles, tags, names: dict[int, str] | None = None) -> None:
    """Write an ASCII MSH 2.2 surface mesh (used by the synthetic generators and tests)."""
    points = np.asarray(points, dtype=np.float64)
    triangles = np.asarray(triangles, dtype=np.int64)
    tags = np.asarray(tags, dtype=np.int64)
    out = ["$MeshFormat", "2.2 0 8", "$EndMeshFormat"]
    if names:
        out += ["$PhysicalNames", str(len(names))]
        out += [f'2 {int(t)} "{n}"' for t, n in sorted(names.items())]
        out += ["$EndPhysicalNames"]
    out += ["$Nodes", str(points.shape[0])]
    # repr of a Python float round-trips exactly (NumPy 2 scalars would print as "np.float64(...)")
    out += [f"{i + 1} {float(p[0])!r} {float(p[1])!r} {float(p[2])!r}" for i, p in enumerate(points)]
    out += ["$EndNodes", "$Elements", str(triangles.shape[0])]
    out += [
        f"{i + 1} 2 2 {int(tags[i])} {int(tags[i])} {t[0] + 1} {t[1] + 1} {t[2] + 1}"
        for i, t in enumerate(triangles)
    ]
    out += ["$EndElements", ""]
    Path(path).write_text("\n".join(out), encoding="utf-8")


# --------------------------------------------------------------------------- #
# Mesh conditioning and checks
# --------------------------------------------------------------------------- #
def merge_duplicate_vertices(verts, tris, tol: float):
    """Merge vertices that round to the same ``tol`` lattice cell (``mesh.py:387-408``).

    Vertex order is unchanged when nothing merges; otherwise vertices follow
    the sorted order of their lattice keys, as in the reference.
    """
    if tol <= 0 or len(verts) == 0:
        return verts, tris, 0
    keys = np.round(verts / tol).astype(np.int64)
    _, first, inverse = np.unique(keys, axis=0, return_index=True, return_inverse=True)
    if len(first) == len(verts):
        return verts, tris, 0
    inverse = np.asarray(inverse).reshape(-1)
    return verts[first], inverse[tris].astype(np.int32), len(verts) - len(first)


def signed_volume_indicator(verts, tris) -> float:
    """``sum p0 . (p1 x p2)``: positive for an outward-wound closed surface (``mesh.py:454-460``)."""
    p0, p1, p2 = verts[tris[:, 0]], verts[tris[:, 1]], verts[tris[:, 2]]
    return float(np.sum(p0 * np.cross(p1, p2)))


def _check_winding(verts, tris, *, repair: bool, aperture_tag: int | None) -> None:
    vol = signed_volume_indicator(verts, tris)
    if aperture_tag is not None:
        if vol <= 0:
            return
        raise MeshError(
            "Coupled infinite-baffle mesh winding appears inverse "
            f"(aperture_tag={aperture_tag}, signed volume positive). "
            "Coupled IB meshes are interior-domain surfaces and must keep "
            "negative signed volume with the aperture normals pointing -Z."
        )
    if vol >= 0:
        return
    if repair:
        logger.info("Flipping triangle winding (signed volume negative)")
        tris[:, [1, 2]] = tris[:, [2, 1]]
        return
    raise MeshError(
        "Mesh triangle winding appears inward (signed volume negative). "
        "Canonical meshes must be emitted with outward normals by the mesher; "
        "pass repair_normals=True only for explicit external-mesh compatibility."
    )


def _check_aperture_normals(verts, tris, tags, aperture_tag: int, tolerance: float = 1.0e-6) -> None:
    mask = np.asarray(tags) == int(aperture_tag)
    if not np.any(mask):
        return
    sel = tris[mask]
    cross = np.cross(verts[sel[:, 1]] - verts[sel[:, 0]], verts[sel[:, 2]] - verts[sel[:, 0]])
    length = np.linalg.norm(cross, axis=1)
    valid = length > 0.0
    if not np.any(valid):
        raise MeshError("Coupled infinite-baffle aperture contains only degenerate triangles")
    nz = cross[valid, 2] / length[valid]
    bad = nz >= -1.0 + tolerance
    if np.any(bad):
        local = int(np.flatnonzero(valid)[int(np.flatnonzero(bad)[0])])
        first = int(np.flatnonzero(mask)[local])
        raise MeshError(
            "Coupled infinite-baffle aperture normals must point -Z for the "
            "interior-domain BIE; regenerate meshes emitted with the old +Z "
            f"aperture contract (triangle {first}, normal_z={nz[bad][0]:.6g})."
        )


def _coerce_aperture_tag(aperture_tag) -> int | None:
    if aperture_tag is None:
        return None
    if isinstance(aperture_tag, bool) or not isinstance(aperture_tag, Integral) or int(aperture_tag) <= 0:
        raise MeshError("aperture_tag must be a positive int or None")
    return int(aperture_tag)


def resolve_aperture_tag(tags, names: dict[int, str], aperture_tag) -> int | None:
    """Aperture tag: explicit, else a group named ``mouth_aperture``, else tag 12 (``mesh.py:487-506``)."""
    present = {int(t) for t in np.unique(tags)}
    explicit = _coerce_aperture_tag(aperture_tag)
    if explicit is not None:
        return explicit if explicit in present else None
    for tag, name in names.items():
        if str(name).strip().lower() == CANONICAL_APERTURE_NAME:
            return int(tag) if int(tag) in present else None
    return CANONICAL_APERTURE_TAG if CANONICAL_APERTURE_TAG in present else None


def _check_groups(tags, aperture_tag: int | None) -> None:
    unique = np.unique(tags)
    candidates = unique if aperture_tag is None else unique[unique != int(aperture_tag)]
    if not np.any(candidates >= 2):
        raise MeshError(f"No velocity source (tag >= 2) found. Tags: {unique.tolist()}")
    if not np.any(unique == 1):
        logger.warning("No rigid wall (tag 1) in mesh")


def open_boundary_edges(triangles_nx3) -> NDArray[np.int32]:
    """Sorted vertex pairs of edges used by exactly one triangle."""
    tris = np.asarray(triangles_nx3)
    if tris.size == 0:
        return np.empty((0, 2), dtype=np.int32)
    edges = np.sort(np.concatenate((tris[:, [0, 1]], tris[:, [1, 2]], tris[:, [2, 0]])), axis=1)
    uniq, counts = np.unique(edges, axis=0, return_counts=True)
    return np.ascontiguousarray(uniq[counts == 1], dtype=np.int32)


def _edges_on_plane(verts, edges, component: int, tol: float):
    return np.all(np.abs(verts[edges, component]) <= tol, axis=1)


def detect_reduced_symmetry_plane(vertices_nx3, triangles_nx3, *, tolerance: float = SYMMETRY_SNAP_TOLERANCE):
    """Conservative guess of the mirror plane(s) of a reduced mesh (``mesh.py:219-276``)."""
    verts = np.asarray(vertices_nx3, dtype=np.float64)
    tris = np.asarray(triangles_nx3, dtype=np.int32)
    if verts.ndim != 2 or verts.shape[1] != 3 or tris.size == 0:
        return None
    used = np.unique(tris.reshape(-1))
    if used.size == 0:
        return None
    edges = open_boundary_edges(tris)
    if edges.size == 0:
        return None
    candidates: dict[str, int] = {}
    for plane, comp in (("yz", 0), ("xz", 1), ("xy", 2)):
        vals = verts[used, comp]
        if (
            np.min(vals) >= -tolerance
            and np.max(vals) > tolerance
            and int(np.count_nonzero(np.abs(vals) <= tolerance)) >= 2
            and int(np.count_nonzero(_edges_on_plane(verts, edges, comp, tolerance))) >= 2
        ):
            candidates[plane] = comp
    for plane, comp in candidates.items():
        if np.all(_edges_on_plane(verts, edges, comp, tolerance)):
            return plane
    if "yz" in candidates and "xz" in candidates:
        explained = _edges_on_plane(verts, edges, 0, tolerance) | _edges_on_plane(verts, edges, 1, tolerance)
        if np.all(explained):
            return "yz+xz"
    return None


def triangle_areas(verts, tris) -> NDArray[np.float64]:
    p0, p1, p2 = verts[tris[:, 0]], verts[tris[:, 1]], verts[tris[:, 2]]
    return np.ascontiguousarray(0.5 * np.linalg.norm(np.cross(p1 - p0, p2 - p0), axis=1))


def make_pure_grid(vertices_nx3, triangles_nx3) -> PureGrid:
    verts = np.asarray(vertices_nx3, dtype=np.float64)
    tris = np.asarray(triangles_nx3, dtype=np.int32)
    return PureGrid(
        vertices=np.ascontiguousarray(verts.T),
        elements=np.ascontiguousarray(tris.T),
        volumes=triangle_areas(verts, tris),
    )


def make_pure_function_spaces(grid) -> tuple[PureFunctionSpace, PureFunctionSpace]:
    """P1 (vertex dofs) and DP0 (triangle dofs) spaces of a grid."""
    if not hasattr(grid, "elements") or not hasattr(grid, "vertices"):
        raise MeshError("Pure function spaces require grid.vertices and grid.elements")
    elements = np.asarray(grid.elements, dtype=np.int32)
    vertices = np.asarray(grid.vertices)
    if elements.ndim != 2 or elements.shape[0] != 3:
        raise MeshError(f"grid.elements must have shape (3, n_triangles), got {elements.shape}")
    if vertices.ndim != 2 or vertices.shape[0] != 3:
        raise MeshError(f"grid.vertices must have shape (3, n_vertices), got {vertices.shape}")
    p1 = PureFunctionSpace(np.ascontiguousarray(elements.T), int(vertices.shape[1]))
    dp0 = PureFunctionSpace(
        np.arange(elements.shape[1], dtype=np.int32)[:, None], int(elements.shape[1])
    )
    return p1, dp0


def mesh_from_arrays(
    vertices_nx3,
    triangles_nx3,
    physical_tags,
    *,
    physical_groups: dict[int, str] | None = None,
) -> LoadedMesh:
    """Wrap in-memory arrays as a ``LoadedMesh`` without file I/O or checks."""
    verts = np.asarray(vertices_nx3, dtype=np.float64)
    tris = np.asarray(triangles_nx3, dtype=np.int32)
    tags = np.asarray(physical_tags, dtype=np.int32).reshape(-1)
    info = MeshInfo(
        n_vertices=int(verts.shape[0]),
        n_triangles=int(tris.shape[0]),
        physical_groups=dict(physical_groups or {}),
        bounding_box_m=(verts.min(axis=0), verts.max(axis=0)),
    )
    return LoadedMesh(grid=make_pure_grid(verts, tris), physical_tags=tags, info=info)


def load_mesh(
    path: str | Path,
    scale: float = 1.0,
    validate: bool = True,
    merge_tol: float = 1e-9,
    repair_normals: bool = False,
    native_symmetry_plane: str | None = None,
    aperture_tag: int | None = None,
) -> LoadedMesh:
    """Load a Gmsh ``.msh`` surface mesh with physical-group tags."""
    path = Path(path)
    if not path.exists():
        raise MeshError(f"Mesh file not found: {path}")
    pts, tris, tags, names = read_gmsh(path)
    verts = pts * scale
    verts, tris, merged = merge_duplicate_vertices(verts, tris, merge_tol)
    if merged:
        logger.info("Merged %d duplicate seam vertices", merged)
    keep = ~((tris[:, 0] == tris[:, 1]) | (tris[:, 1] == tris[:, 2]) | (tris[:, 0] == tris[:, 2]))
    if not np.all(keep):
        logger.info("Removed %d degenerate triangles", int(np.sum(~keep)))
        tris, tags = tris[keep], tags[keep]
    tris = np.ascontiguousarray(tris, dtype=np.int32)
    ap = resolve_aperture_tag(tags, names, aperture_tag)
    if validate:
        _check_winding(verts, tris, repair=repair_normals, aperture_tag=ap)
        if ap is not None:
            _check_aperture_normals(verts, tris, tags, ap)
        _check_groups(tags, ap)
    if native_symmetry_plane is None:
        suspected = detect_reduced_symmetry_plane(verts, tris)
        if suspected is not None:
            warnings.warn(
                "Mesh may be a reduced native-symmetry mesh "
                f"(suspected plane {suspected!r}) but native_symmetry_plane is None; "
                "if this is intended as a mirror-reduced mesh, pass "
                f"native_symmetry_plane={suspected!r} in SolveConfig to solve the "
                "free-space mirrored geometry. If the rim is a real open boundary, "
                "ignore this warning.",
                RuntimeWarning,
                stacklevel=2,
            )
    return mesh_from_arrays(verts, tris, tags, physical_groups=names)
