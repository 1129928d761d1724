"""Neumann data, source velocity profiles and surface-pressure reductions.

Restates ``hornlab_metal_bem/bie.py`` of the reference:

* DP0 Neumann data ``q = i rho omega v_n`` per driven face, with
  ``v_n = w`` (VELOCITY) or ``w / (i omega)`` (ACCELERATION), tags carrying a
  Robin admittance skipped (``bie.py:287-362``);
* per-face source multipliers for normal / axial / taper / annular / per-face
  / callable profiles, each axial projection oriented outward-positive per tag
  by its area-weighted sign (``bie.py:154-284``);
* host twins of the area-weighted tag pressure averages (``bie.py:365-434``);
  the GPU path computes the same reductions on the device.
"""
from __future__ import annotations

import numpy as np
from numpy.typing import NDArray

from .config import (
    AnnularProfile,
    AxialProfile,
    CallableProfile,
    NormalProfile,
    PerFaceProfile,
    SolveConfig,
    SourceMotion,
    TaperProfile,
    VelocityMode,
)


def _unit_axis(axis) -> NDArray[np.float64] | None:
    a = np.asarray(axis, dtype=np.float64).reshape(-1)
    if a.shape[0] != 3:
        return None
    n = float(np.linalg.norm(a))
    if not np.isfinite(n) or n <= 1e-12:
        return None
    return a / n


def _face_geometry(grid):
    verts = np.asarray(grid.vertices.T, dtype=np.float64)
    tris = np.asarray(grid.elements.T, dtype=np.int32)
    p0, p1, p2 = verts[tris[:, 0]], verts[tris[:, 1]], verts[tris[:, 2]]
    cross = np.cross(p1 - p0, p2 - p0)
    mag = np.linalg.norm(cross, axis=1)
    return cross, mag, (p0 + p1 + p2) / 3.0


def _oriented_projection(cross, mag, faces, axis) -> NDArray[np.float64]:
    m = mag[faces]
    unit = cross[faces] / np.where(m > 1e-15, m, 1.0)[:, None]
    proj = unit @ axis
    return -proj if float(proj @ m) < 0.0 else proj


def _normalised_radius(centroids, faces, axis, center) -> NDArray[np.float64]:
    d = centroids[faces] - center[None, :]
    radial = np.linalg.norm(d - np.outer(d @ axis, axis), axis=1)
    rmax = float(np.max(radial)) if radial.size else 0.0
    if not np.isfinite(rmax) or rmax <= 1e-15:
        return np.zeros_like(radial)
    return np.clip(radial / rmax, 0.0, 1.0)


def _taper(t, profile: TaperProfile) -> NDArray[np.float64]:
    out = np.ones_like(t)
    ramp = t > profile.start
    if np.any(ramp):
        x = np.clip((t[ramp] - profile.start) / (1.0 - profile.start), 0.0, 1.0)
        out[ramp] = 1.0 - x if profile.kind == "linear" else 0.5 * (1.0 + np.cos(np.pi * x))
    out[t >= 1.0] = 0.0
    return out


def profile_for_tag(config: SolveConfig, tag: int):
    profiles = {int(k): v for k, v in (config.source_velocity_profiles or {}).items()}
    if tag in profiles:
        return profiles[tag]
    return AxialProfile() if config.source_motion == SourceMotion.AXIAL else NormalProfile()


def build_source_face_scale(grid, physical_tags, config: SolveConfig, axis, source_center):
    """Per-face source multiplier, or ``None`` when every driven tag is plain normal."""
    profiles = {int(k): v for k, v in (config.source_velocity_profiles or {}).items()}
    tags_used = sorted({int(t) for t in config.velocity_sources} | set(profiles))
    if not tags_used:
        return None
    eff = {t: profile_for_tag(config, t) for t in tags_used}
    if all(isinstance(p, NormalProfile) for p in eff.values()):
        return None
    unit = _unit_axis(axis)
    if unit is None and all(isinstance(p, (NormalProfile, AxialProfile)) for p in eff.values()):
        return None
    if unit is None and any(isinstance(p, (TaperProfile, AnnularProfile, CallableProfile)) for p in eff.values()):
        raise ValueError("source velocity profiles require a non-degenerate axis")
    center = np.asarray(source_center, dtype=np.float64).reshape(-1)
    if center.shape[0] != 3:
        raise ValueError("source_center must have shape (3,)")

    cross, mag, centroids = _face_geometry(grid)
    unit_normals = cross / np.where(mag > 1e-15, mag, 1.0)[:, None]
    tags = np.asarray(physical_tags)
    scale = np.zeros(tags.shape[0], dtype=np.complex128)
    any_face = False
    is_complex = False
    for tag in tags_used:
        faces = np.flatnonzero(tags == tag)
        if faces.size == 0:
            continue
        any_face = True
        p = eff[tag]
        if isinstance(p, NormalProfile):
            vals = np.ones(faces.size)
        elif isinstance(p, AxialProfile):
            vals = np.ones(faces.size) if unit is None else _oriented_projection(cross, mag, faces, unit)
        elif isinstance(p, TaperProfile):
            vals = _oriented_projection(cross, mag, faces, unit) * _taper(
                _normalised_radius(centroids, faces, unit, center), p
            )
        elif isinstance(p, AnnularProfile):
            t = _normalised_radius(centroids, faces, unit, center)
            vals = _oriented_projection(cross, mag, faces, unit) * ((t >= p.r_inner) & (t <= p.r_outer))
        elif isinstance(p, PerFaceProfile):
            vals = np.asarray(p.weights, dtype=np.complex128)
            if vals.ndim != 1 or vals.shape[0] != faces.size:
                raise ValueError(
                    f"PerFaceProfile.weights length must equal the number of faces for tag {tag}"
                )
            if not np.all(np.isfinite(vals)):
                raise ValueError("PerFaceProfile.weights must be finite")
            is_complex |= bool(np.any(vals.imag != 0.0))
        elif isinstance(p, CallableProfile):
            vals = np.asarray(
                p.callback(centroids[faces], unit_normals[faces], unit.copy(), center.copy()),
                dtype=np.complex128,
            )
            if vals.ndim != 1 or vals.shape[0] != faces.size:
                raise ValueError(f"CallableProfile.callback must return one weight per face for tag {tag}")
            if not np.all(np.isfinite(vals)):
                raise ValueError("CallableProfile.callback returned non-finite weights")
            is_complex |= bool(np.any(vals.imag != 0.0))
        else:  # pragma: no cover - config validation rejects this
            raise ValueError("source_velocity_profiles values must be SourceProfile instances")
        scale[faces] = vals
    if not any_face:
        return None
    return scale if is_complex else scale.real.astype(np.float64, copy=False)


def build_driver_neumann(
    n_faces: int,
    physical_tags,
    omega: float,
    config: SolveConfig,
    dtype=np.complex64,
    impedance_tags: set[int] | None = None,
    source_face_scale=None,
) -> NDArray:
    """DP0 Neumann coefficients ``q_tau = i rho omega v_n(tau)`` at one angular frequency."""
    q = np.zeros(n_faces, dtype=dtype)
    freq_hz = float(omega) / (2.0 * np.pi) if omega > 0 else 0.0
    sources = (
        config.velocity_source_callback(freq_hz)
        if config.velocity_source_callback is not None
        else config.velocity_sources
    )
    if impedance_tags is None:
        impedance_tags = set(config.impedance_sources.keys())
        if config.impedance_source_callback is not None:
            impedance_tags |= {int(t) for t in config.impedance_source_callback(freq_hz)}
    tags = np.asarray(physical_tags)
    accel = config.velocity_mode == VelocityMode.ACCELERATION
    for tag, weight in sources.items():
        if tag in impedance_tags:
            continue
        faces = np.flatnonzero(tags == tag)
        if faces.size == 0:
            continue
        if source_face_scale is None:
            vn = weight
            if accel:
                vn = weight / (1j * omega) if omega > 0 else 0.0
        else:
            vn = weight * source_face_scale[faces]
            if accel:
                vn = vn / (1j * omega) if omega > 0 else np.zeros_like(vn)
        q[faces] = 1j * config.air_density * omega * vn
    return q


def tag_average_pressure(areas, local2global, physical_tags, p1_coeffs, tag: int) -> complex:
    """``integral(p dA) / integral(dA)`` over faces of ``tag`` with p = mean of the three P1 values."""
    faces = np.flatnonzero(np.asarray(physical_tags) == tag)
    if faces.size == 0:
        return 0.0 + 0.0j
    a = np.asarray(areas)[faces]
    pavg = np.mean(np.asarray(p1_coeffs)[np.asarray(local2global)[faces]], axis=1)
    total = np.sum(a)
    if abs(total) < 1e-30:
        return 0.0 + 0.0j
    return complex(np.sum(pavg * a) / total)


def compute_surface_pressure_avg(areas, local2global, physical_tags, p1_coeffs, tags) -> dict[int, complex]:
    return {int(t): tag_average_pressure(areas, local2global, physical_tags, p1_coeffs, int(t)) for t in tags}
