"""B200-native dense Helmholtz BEM with the public API of ``hornlab_metal_bem``.

Drop-in surface (``hornlab_metal_bem/__init__.py:26-252`` of the reference):
``native_config``, ``solve``, ``solve_frequencies``, ``solve_multi_source``,
``load_mesh``/``LoadedMesh``/``MeshError``, ``SolveConfig``,
``ObservationConfig``, source profiles, ``SolveResult``/``MeshInfo``,
``ObservationFrame``/``infer_frame``.  Assembly, dense LU, field and
reductions run as hand-written sm_100a kernels in ``libhbem.so`` through the C
ABI of ``include/hbem.h``; there is no CPU fallback.

The reference's axisymmetric solver (``solve_circsym*``) is outside this
package's scope and is not exported.
"""
from __future__ import annotations

from dataclasses import replace as _replace

import numpy as np

from .config import (
    AnnularProfile,
    AxialProfile,
    CallableProfile,
    NormalProfile,
    ObservationConfig,
    PerFaceProfile,
    SolveConfig,
    SourceMotion,
    SourceProfile,
    TaperProfile,
    VelocityMode,
)
from .mesh import LoadedMesh, MeshError, load_mesh, mesh_from_arrays
from .observation import ObservationFrame, infer_frame, project_to_symmetry_subspace
from .result import MeshInfo, SolveResult

__all__ = [
    "native_config", "solve", "solve_frequencies", "solve_multi_source", "load_mesh", "mesh_from_arrays",
    "SolveConfig", "SolveResult", "ObservationConfig", "VelocityMode", "SourceMotion", "SourceProfile",
    "NormalProfile", "AxialProfile", "TaperProfile", "AnnularProfile", "PerFaceProfile", "CallableProfile",
    "LoadedMesh", "MeshInfo", "MeshError", "ObservationFrame", "infer_frame",
]


def native_config(**overrides) -> SolveConfig:
    """The supported configuration: corrected (Duffy) assembly plus caller overrides."""
    values = {"metal_native_assembly_mode": "corrected"}
    values.update(overrides)
    return SolveConfig(**values)


def _resolve_mesh(mesh, config: SolveConfig) -> LoadedMesh:
    if isinstance(mesh, LoadedMesh):
        return mesh
    return load_mesh(
        mesh, scale=config.mesh_scale, validate=config.mesh_validate, merge_tol=config.mesh_merge_tol,
        repair_normals=config.mesh_repair_normals, native_symmetry_plane=config.native_symmetry_plane,
        aperture_tag=config.aperture_tag,
    )


def _aperture_origin(loaded: LoadedMesh, aperture_tag: int):
    """Area-weighted centroid of the aperture faces (``__init__.py:97-118``)."""
    tags = np.asarray(loaded.physical_tags)
    sel = tags == int(aperture_tag)
    if not np.any(sel):
        return None
    v = np.asarray(loaded.grid.vertices.T, dtype=np.float64)
    f = np.asarray(loaded.grid.elements.T)[sel]
    p0, p1, p2 = v[f[:, 0]], v[f[:, 1]], v[f[:, 2]]
    a = 0.5 * np.linalg.norm(np.cross(p1 - p0, p2 - p0), axis=1)
    ok = a > 1.0e-15
    if not np.any(ok):
        return None
    return np.average((p0[ok] + p1[ok] + p2[ok]) / 3.0, weights=a[ok], axis=0)


def _resolve_frame(loaded: LoadedMesh, config: SolveConfig) -> ObservationFrame:
    if config.frame_override is not None:
        return config.frame_override
    frame = infer_frame(
        loaded.grid, loaded.physical_tags, source_tag=min(config.velocity_sources.keys(), default=2),
        origin_at=config.observation.origin, symmetry_plane=config.native_symmetry_plane,
    )
    if config.aperture_tag is not None and config.observation.origin == "mouth":
        origin = _aperture_origin(loaded, config.aperture_tag)
        if origin is not None:
            origin = project_to_symmetry_subspace(origin, config.native_symmetry_plane)
            frame = _replace(frame, origin=origin, mouth_center=origin)
    return frame


def solve(mesh, config: SolveConfig | None = None) -> SolveResult:
    """Frequency sweep of ``config``'s grid on the GPU."""
    from .sweep import build_frequency_grid, run_sweep, should_route_native

    config = config or native_config()
    loaded = _resolve_mesh(mesh, config)
    frame = _resolve_frame(loaded, config)
    should_route_native(config)
    return run_sweep(loaded, build_frequency_grid(config), frame, config)


def solve_frequencies(mesh, frequencies_hz, config: SolveConfig | None = None) -> SolveResult:
    """Sweep at caller-ordered frequencies."""
    from .sweep import run_sweep, should_route_native

    config = config or native_config()
    loaded = _resolve_mesh(mesh, config)
    frame = _resolve_frame(loaded, config)
    should_route_native(config)
    return run_sweep(loaded, np.asarray(frequencies_hz, dtype=np.float64), frame, config)


def solve_multi_source(mesh, sources: list[dict[int, complex]], config: SolveConfig | None = None,
                       frequencies_hz=None) -> list[SolveResult]:
    """One ``SolveResult`` per velocity-source dict, sharing the mesh session and frame."""
    from .sweep import build_frequency_grid, run_sweep_multi_source, should_route_native

    config = config or native_config()
    if not sources:
        raise ValueError("sources must contain at least one velocity dict")
    loaded = _resolve_mesh(mesh, config)
    frame = _resolve_frame(loaded, _replace(config, velocity_sources=dict(sources[0])))
    freqs = build_frequency_grid(config) if frequencies_hz is None else np.asarray(frequencies_hz, dtype=np.float64)
    should_route_native(config)
    return run_sweep_multi_source(loaded, freqs, frame, config, sources)
