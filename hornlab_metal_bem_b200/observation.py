"""Radiation frame inference and polar observation arcs.

Restates ``hornlab_metal_bem/observation.py:76-313`` of the reference:

* the forward axis is the area-weighted, hemisphere-aligned sum of the source
  tag's face normals (PCA of the vertex cloud when that is degenerate),
  projected onto the symmetry subspace for mirror-reduced meshes;
* the axis is flipped so the source sits at the minimum projection, unless the
  source is buried mid-span (> 25 % from both extremes, an enclosure), in
  which case the source normal is trusted as is;
* the mouth centre is the mean of the vertices within 2 % of the span from
  the forward extreme; transverse vectors come from Gram-Schmidt against +X
  (or +Y when the axis is within ~26 deg of X);
* arcs are ``origin + r (cos t * axis + sin t * transverse)`` per plane.
"""
from __future__ import annotations

import logging
from dataclasses import dataclass

import numpy as np
from numpy.typing import NDArray

from .config import ObservationConfig

logger = logging.getLogger(__name__)


@dataclass
class ObservationFrame:
    axis: NDArray[np.float64]
    origin: NDArray[np.float64]
    u: NDArray[np.float64]
    v: NDArray[np.float64]
    mouth_center: NDArray[np.float64]
    source_center: NDArray[np.float64]


def project_to_symmetry_subspace(vector, symmetry_plane: str | None) -> NDArray[np.float64]:
    """Zero the components normal to the requested mirror planes."""
    out = np.array(vector, dtype=np.float64, copy=True)
    if symmetry_plane is None:
        return out
    plane = str(symmetry_plane).strip().lower()
    zero = {"yz": (0,), "xz": (1,), "yz+xz": (0, 1), "xy": (2,)}.get(plane, ())
    for comp in zero:
        out[comp] = 0.0
    return out


def _pca_axis(vertices: NDArray[np.float64], center: NDArray[np.float64]) -> NDArray[np.float64]:
    d = vertices - center[None, :]
    if d.shape[0] == 0:
        return np.array([0.0, 1.0, 0.0])
    w, vecs = np.linalg.eigh(d.T @ d)
    axis = np.asarray(vecs[:, int(np.argmax(w))], dtype=np.float64)
    nrm = float(np.linalg.norm(axis))
    return np.array([0.0, 1.0, 0.0]) if nrm <= 1e-12 else axis / nrm


def infer_frame(
    grid,
    physical_tags,
    source_tag: int = 2,
    origin_at: str = "mouth",
    symmetry_plane: str | None = None,
) -> ObservationFrame:
    vertices = np.array(grid.vertices.T, dtype=np.float64)
    elements = np.array(grid.elements.T, dtype=np.int32)
    tags = np.asarray(physical_tags)
    sel = tags == source_tag
    if not np.any(sel):
        raise ValueError(f"No elements with tag {source_tag} in mesh")
    src = elements[sel]
    src = src[np.all((src >= 0) & (src < vertices.shape[0]), axis=1)]

    normal_dir = None
    source_center = np.mean(vertices, axis=0)
    if src.shape[0] > 0:
        p0, p1, p2 = vertices[src[:, 0]], vertices[src[:, 1]], vertices[src[:, 2]]
        cross = np.cross(p1 - p0, p2 - p0)
        mag = np.linalg.norm(cross, axis=1)
        ok = mag > 1e-15
        if np.any(ok):
            cross, mag = cross[ok], mag[ok]
            centroids = (p0[ok] + p1[ok] + p2[ok]) / 3.0
            sign = np.sign(cross @ cross[0])
            sign[sign == 0] = 1.0
            total = np.sum(cross * sign[:, None], axis=0)
            tn = float(np.linalg.norm(total))
            if tn > 1e-12:
                normal_dir = total / tn
                source_center = np.average(centroids, weights=mag, axis=0)
    from_tags = normal_dir is not None
    if normal_dir is None:
        normal_dir = _pca_axis(vertices, source_center)

    if symmetry_plane is not None:
        proj = project_to_symmetry_subspace(normal_dir, symmetry_plane)
        pn = float(np.linalg.norm(proj))
        if pn > 1e-12:
            normal_dir = proj / pn

    heights = vertices @ normal_dir
    s = source_center @ normal_dir
    hi, lo = heights.max(), heights.min()
    span = hi - lo
    if span < 1e-12:
        axis = normal_dir.copy()
    else:
        frac_lo = abs(s - lo) / span
        frac_hi = abs(s - hi) / span
        if from_tags and min(frac_lo, frac_hi) > 0.25:
            axis = normal_dir.copy()
            logger.info("Enclosed geometry detected (source at %.0f%% of span)", 100 * frac_lo)
        elif frac_lo < frac_hi:
            axis = normal_dir.copy()
        else:
            axis = -normal_dir

    along = vertices @ axis
    cut = along.max() - 0.02 * (along.max() - along.min())
    mouth_center = vertices[along >= cut].mean(axis=0)

    ex = np.array([1.0, 0.0, 0.0])
    ey = np.array([0.0, 1.0, 0.0])
    ref = ex if abs(float(axis @ ex)) < 0.9 else ey
    u = ref - float(ref @ axis) * axis
    u /= np.linalg.norm(u)
    v = np.cross(axis, u)

    origin = mouth_center.copy() if origin_at == "mouth" else source_center.copy()
    if symmetry_plane is not None:
        origin = project_to_symmetry_subspace(origin, symmetry_plane)
    return ObservationFrame(axis=axis, origin=origin, u=u, v=v, mouth_center=mouth_center, source_center=source_center)


def build_observation_points(frame: ObservationFrame, config: ObservationConfig):
    """Return ``(points (P, N, 3), angles_deg (N,))``."""
    angles = np.linspace(config.angle_min_deg, config.angle_max_deg, config.angle_count)
    if config.custom_points is not None:
        blocks = []
        for plane in config.planes:
            if plane not in config.custom_points:
                raise ValueError(
                    f"custom_points missing plane {plane!r}; available: {list(config.custom_points.keys())}"
                )
            pts = np.asarray(config.custom_points[plane], dtype=np.float64)
            if pts.ndim != 2 or pts.shape[1] != 3:
                raise ValueError(f"custom_points[{plane!r}] must be (N, 3), got {pts.shape}")
            blocks.append(pts)
        counts = [b.shape[0] for b in blocks]
        if len(set(counts)) > 1:
            raise ValueError(
                "All custom_points planes must have the same number of points, "
                f"got {dict(zip(config.planes, counts))}"
            )
        if counts[0] != config.angle_count:
            angles = np.linspace(config.angle_min_deg, config.angle_max_deg, counts[0])
        return np.stack(blocks, axis=0), angles

    theta = np.deg2rad(angles)
    r = config.distance_m
    blocks = []
    for plane in config.planes:
        if plane == "horizontal":
            t = frame.u
        elif plane == "vertical":
            t = frame.v
        elif plane == "diagonal":
            t = (frame.u + frame.v) / np.sqrt(2)
        else:
            raise ValueError(f"Unknown plane: {plane!r}")
        blocks.append(
            frame.origin[None, :]
            + r * np.cos(theta)[:, None] * frame.axis[None, :]
            + r * np.sin(theta)[:, None] * t[None, :]
        )
    return np.stack(blocks, axis=0), angles
