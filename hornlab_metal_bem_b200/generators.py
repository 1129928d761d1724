"""Synthetic surface meshes standing in for the reference's production meshes.

The reference quotes its numbers on HornLab production meshes (ASRO2) that are
not distributed; these seeded generators produce meshes with the same shapes,
sizes and tag conventions (tag 2 = driven source, tag 1 = rigid wall):

* ``icosphere``: subdivided icosahedron on a sphere (pulsating-sphere case).
* ``horn``: closed body of revolution made of a driver can (rear disc + short
  cylinder), an outer wall, a mouth lip, a flared inner wall and the throat
  disc (tag 2).  The flare is ``r(z) = r_t + (r_m - r_t)(e^{m z} - 1)/(e^{m L} - 1)``:
  a pure exponential cannot meet both radii for an arbitrary flare constant
  ``m``, so ``m`` is a shape parameter and both radii are met exactly.  The
  mesh can be the full revolution or the ``x >= 0, y >= 0`` quarter for the
  ``yz+xz`` image method.

Every mesh is wound outward (positive signed-volume indicator).
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from .mesh import LoadedMesh, mesh_from_arrays


# --------------------------------------------------------------------------- #
# Icosphere
# --------------------------------------------------------------------------- #
def icosphere(level: int = 3, radius: float = 0.1, tag: int = 2) -> LoadedMesh:
    """Icosahedron refined ``level`` times (10 * 4**level + 2 vertices)."""
    t = (1.0 + math.sqrt(5.0)) / 2.0
    verts = [
        (-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0),
        (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
        (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1),
    ]
    faces = [
        (0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11),
        (1, 5, 9), (5, 11, 4), (11, 10, 2), (10, 7, 6), (7, 1, 8),
        (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9),
        (4, 9, 5), (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1),
    ]
    pts = [np.asarray(v, dtype=np.float64) / np.linalg.norm(v) for v in verts]
    for _ in range(level):
        cache: dict[tuple[int, int], int] = {}

        def mid(a: int, b: int) -> int:
            key = (a, b) if a < b else (b, a)
            if key not in cache:
                m = pts[a] + pts[b]
                pts.append(m / np.linalg.norm(m))
                cache[key] = len(pts) - 1
            return cache[key]

        nxt = []
        for a, b, c in faces:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nxt += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = nxt
    v = np.asarray(pts) * radius
    f = np.asarray(faces, dtype=np.int32)
    return mesh_from_arrays(v, f, np.full(f.shape[0], tag, dtype=np.int32), physical_groups={tag: "sphere"})


# --------------------------------------------------------------------------- #
# Bodies of revolution
# --------------------------------------------------------------------------- #
def _ring_angles(r: float, h: float, phi_max: float) -> np.ndarray:
    if r <= 1e-12:
        return np.zeros(1)
    n = max(1, int(math.ceil(r * phi_max / h)))
    if phi_max >= 2 * math.pi - 1e-12:
        n = max(n, 3)
        return np.linspace(0.0, phi_max, n, endpoint=False)
    return np.linspace(0.0, phi_max, n + 1)


def revolve(profile_rz, tags_seg, h: float, quarter: bool, half: bool = False) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """Mesh the surface swept by a meridian polyline ``(r, z)`` around the z axis.

    ``tags_seg[i]`` tags the strip between profile nodes ``i`` and ``i + 1``.
    Points with ``r == 0`` collapse to one vertex on the axis.  Strip sides
    are wound so that the normal points to the left of the direction of
    travel along the profile in the (r, z) half-plane, i.e. consistently for
    a profile that runs clockwise around the body's meridian section.
    """
    # sector: quarter x, y >= 0 (yz + xz planes); half x >= 0 (yz plane), swept
    # from -pi/2 to pi/2; else the full revolution
    phi_max = 0.5 * math.pi if quarter else (math.pi if half else 2.0 * math.pi)
    phi0 = -0.5 * math.pi if (half and not quarter) else 0.0
    closed = not (quarter or half)
    verts: list[tuple[float, float, float]] = []
    rings: list[tuple[np.ndarray, list[int]]] = []
    for r, z in profile_rz:
        ang = _ring_angles(float(r), h, phi_max)
        ids = []
        for a in ang:
            x, y = float(r) * math.cos(a + phi0), float(r) * math.sin(a + phi0)
            if quarter:
                if abs(a - phi_max) < 1e-12:
                    x = 0.0
                if a == 0.0:
                    y = 0.0
            elif half and (a == 0.0 or abs(a - phi_max) < 1e-12):
                x = 0.0
            ids.append(len(verts))
            verts.append((x, y, float(z)))
        rings.append((ang, ids))

    tris: list[tuple[int, int, int]] = []
    tags: list[int] = []

    def add(a: int, b: int, c: int, tag: int) -> None:
        tris.append((a, b, c))
        tags.append(tag)

    for s in range(len(rings) - 1):
        (aa, ia), (ab, ib) = rings[s], rings[s + 1]
        tag = int(tags_seg[s])
        if len(ia) == 1 and len(ib) == 1:
            continue
        if len(ia) == 1 or len(ib) == 1:
            apex_first = len(ia) == 1
            apex = ia[0] if apex_first else ib[0]
            ring = ib if apex_first else ia
            m = len(ring) if closed else len(ring) - 1
            for j in range(m):
                p, q = ring[j], ring[(j + 1) % len(ring)]
                if apex_first:
                    add(apex, q, p, tag)
                else:
                    add(apex, p, q, tag)
            continue
        # zip two rings by angle
        na, nb = len(ia), len(ib)
        ea = na if closed else na - 1
        eb = nb if closed else nb - 1
        i = j = 0
        while i < ea or j < eb:
            ta = aa[i + 1] if i + 1 < na else phi_max
            tb = ab[j + 1] if j + 1 < nb else phi_max
            a0, a1 = ia[i % na], ia[(i + 1) % na]
            b0, b1 = ib[j % nb], ib[(j + 1) % nb]
            if j >= eb or (i < ea and ta <= tb):
                add(a0, a1, b0, tag)
                i += 1
            else:
                add(a0, b1, b0, tag)
                j += 1
    v = np.asarray(verts, dtype=np.float64)
    f = np.asarray(tris, dtype=np.int32)
    return v, f, np.asarray(tags, dtype=np.int32)


def _orient_outward(v: np.ndarray, f: np.ndarray) -> np.ndarray:
    p0, p1, p2 = v[f[:, 0]], v[f[:, 1]], v[f[:, 2]]
    if float(np.sum(p0 * np.cross(p1, p2))) < 0:
        f = f[:, [0, 2, 1]]
    return np.ascontiguousarray(f)


@dataclass(frozen=True)
class HornSpec:
    throat_radius: float = 0.0127
    mouth_radius: float = 0.150
    length: float = 0.120
    flare: float = 20.6
    lip: float = 0.005
    can_depth: float = 0.020
    edge: float = 0.008


def horn_spec_from_seed(seed: int, *, edge: float, flare_range=(10.0, 40.0), mouth_range=None,
                        lip_range=(0.003, 0.008), **fixed) -> HornSpec:
    """Draw the flare constant, lip thickness (and optionally mouth radius) from ``seed``."""
    rng = np.random.default_rng(seed)
    flare = float(rng.uniform(*flare_range))
    lip = float(rng.uniform(*lip_range))
    mouth = float(rng.uniform(*mouth_range)) if mouth_range is not None else fixed.pop("mouth_radius", 0.150)
    return HornSpec(mouth_radius=mouth, flare=flare, lip=lip, edge=edge, **fixed)


def horn_profile(spec: HornSpec) -> tuple[np.ndarray, np.ndarray]:
    """Meridian polyline (r, z) of the closed horn body and per-segment tags."""
    h = spec.edge
    L, rt, rm, m = spec.length, spec.throat_radius, spec.mouth_radius, spec.flare

    def flare_r(z):
        return rt + (rm - rt) * (np.expm1(m * z) / np.expm1(m * L))

    def seg(p0, p1):
        n = max(1, int(math.ceil(math.dist(p0, p1) / h)))
        return [(p0[0] + (p1[0] - p0[0]) * t, p0[1] + (p1[1] - p0[1]) * t) for t in np.linspace(0, 1, n + 1)]

    def curve(fr, z0, z1, offset):
        zs = np.linspace(z0, z1, 4000)
        rs = fr(zs) + offset
        ds = np.concatenate([[0.0], np.cumsum(np.hypot(np.diff(rs), np.diff(zs)))])
        n = max(1, int(math.ceil(ds[-1] / h)))
        s = np.linspace(0, ds[-1], n + 1)
        return list(zip(np.interp(s, ds, rs), np.interp(s, ds, zs)))

    t = spec.lip
    r_can = rt + t
    pts: list[tuple[float, float]] = []
    tags: list[int] = []

    def extend(points, tag):
        start = 1 if pts else 0
        for p in points[start:]:
            if pts:
                tags.append(tag)
            pts.append((float(p[0]), float(p[1])))

    extend(seg((0.0, -spec.can_depth), (r_can, -spec.can_depth)), 1)     # rear disc
    extend(seg((r_can, -spec.can_depth), (r_can, 0.0)), 1)                # can side
    extend(curve(flare_r, 0.0, L, t), 1)                                  # outer wall
    extend(seg((rm + t, L), (rm, L)), 1)                                  # lip
    extend(curve(flare_r, L, 0.0, 0.0), 1)                                # inner wall
    extend(seg((rt, 0.0), (0.0, 0.0)), 2)                                 # throat disc (source)
    return np.asarray(pts), np.asarray(tags, dtype=np.int32)


def horn(spec: HornSpec = HornSpec(), quarter: bool = True, half: bool = False) -> LoadedMesh:
    """Closed round horn: quarter (x, y >= 0; yz + xz planes), half (x >= 0; yz plane) or full."""
    prof, seg_tags = horn_profile(spec)
    v, f, tags = revolve(prof, seg_tags, spec.edge, quarter, half and not quarter)
    # merge duplicate vertices created where the profile revisits a radius
    keys = np.round(v / 1e-9).astype(np.int64)
    _, first, inv = np.unique(keys, axis=0, return_index=True, return_inverse=True)
    inv = np.asarray(inv).reshape(-1)
    order = np.argsort(first)
    remap = np.empty_like(order)
    remap[order] = np.arange(order.size)
    v = v[first[order]]
    f = remap[inv[f]].astype(np.int32)
    keep = ~((f[:, 0] == f[:, 1]) | (f[:, 1] == f[:, 2]) | (f[:, 0] == f[:, 2]))
    f, tags = f[keep], tags[keep]
    if quarter or half:
        p0, p1, p2 = v[f[:, 0]], v[f[:, 1]], v[f[:, 2]]
        n = np.cross(p1 - p0, p2 - p0)
        c = (p0 + p1 + p2) / 3.0
        radial = np.stack([c[:, 0], c[:, 1], np.zeros(len(c))], axis=1)
        # orientation of the quarter: use the full-revolution convention by checking
        # the rear-disc faces, whose outward normal is -z
        rear = np.abs(c[:, 2] + spec.can_depth) < 1e-12
        if np.any(rear) and float(np.mean(n[rear, 2])) > 0:
            f = f[:, [0, 2, 1]]
        del radial
    else:
        f = _orient_outward(v, f)
    return mesh_from_arrays(v, f, tags, physical_groups={1: "wall", 2: "throat"})


def baffled_horn(spec: HornSpec = HornSpec(), quarter: bool = False, aperture_tag: int = 12) -> LoadedMesh:
    """Interior-domain horn for the coupled infinite baffle.

    The cavity is the horn's air volume: throat disc (tag 2) at z = -L, flared
    wall (tag 1) and the flush mouth aperture (``aperture_tag``) at z = 0.
    Normals point into the cavity (aperture normals -Z), so the signed-volume
    indicator is negative, as the reference requires for coupled meshes
    (``mesh.py:411-484``).
    """
    h = spec.edge
    L, rt, rm, m = spec.length, spec.throat_radius, spec.mouth_radius, spec.flare

    def flare_r(z):
        return rt + (rm - rt) * (np.expm1(m * (z + L)) / np.expm1(m * L))

    pts: list[tuple[float, float]] = []
    tags: list[int] = []

    def extend(points, tag):
        start = 1 if pts else 0
        for p in points[start:]:
            if pts:
                tags.append(tag)
            pts.append((float(p[0]), float(p[1])))

    def seg(p0, p1):
        n = max(1, int(math.ceil(math.dist(p0, p1) / h)))
        return [(p0[0] + (p1[0] - p0[0]) * t, p0[1] + (p1[1] - p0[1]) * t) for t in np.linspace(0, 1, n + 1)]

    zs = np.linspace(-L, 0.0, 4000)
    rs = flare_r(zs)
    ds = np.concatenate([[0.0], np.cumsum(np.hypot(np.diff(rs), np.diff(zs)))])
    nseg = max(1, int(math.ceil(ds[-1] / h)))
    sgrid = np.linspace(0, ds[-1], nseg + 1)
    wall = list(zip(np.interp(sgrid, ds, rs), np.interp(sgrid, ds, zs)))
    extend(seg((0.0, -L), (rt, -L)), 2)
    extend(wall, 1)
    extend(seg((rm, 0.0), (0.0, 0.0)), aperture_tag)
    v, f, t = revolve(np.asarray(pts), np.asarray(tags, dtype=np.int32), h, quarter)
    keys = np.round(v / 1e-9).astype(np.int64)
    _, first, inv = np.unique(keys, axis=0, return_index=True, return_inverse=True)
    inv = np.asarray(inv).reshape(-1)
    order = np.argsort(first)
    remap = np.empty_like(order)
    remap[order] = np.arange(order.size)
    v = v[first[order]]
    f = remap[inv[f]].astype(np.int32)
    keep = ~((f[:, 0] == f[:, 1]) | (f[:, 1] == f[:, 2]) | (f[:, 0] == f[:, 2]))
    f, t = f[keep], t[keep]
    # orient so the aperture normals point -Z (into the cavity)
    ap = t == aperture_tag
    p0, p1, p2 = v[f[:, 0]], v[f[:, 1]], v[f[:, 2]]
    nz = np.cross(p1 - p0, p2 - p0)[:, 2]
    if float(np.mean(nz[ap])) > 0:
        f = f[:, [0, 2, 1]]
    return mesh_from_arrays(v, np.ascontiguousarray(f), t,
                            physical_groups={1: "wall", 2: "throat", aperture_tag: "mouth_aperture"})
