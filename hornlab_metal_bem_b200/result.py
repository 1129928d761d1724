"""Solve result containers (field-for-field ``hornlab_metal_bem/result.py:13-64``)."""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Any

import numpy as np
from numpy.typing import NDArray

from .config import SolveConfig


@dataclass
class MeshInfo:
    n_vertices: int
    n_triangles: int
    physical_groups: dict[int, str]
    bounding_box_m: tuple[NDArray[np.float64], NDArray[np.float64]]


@dataclass
class SolveResult:
    """Sweep output.  ``F`` = frequencies, ``P`` = observation planes, ``N`` = angles."""

    frequencies_hz: NDArray[np.float64]
    pressure_complex: NDArray[np.complex128]          # (F, P, N)
    directivity_db: NDArray[np.float64]               # (F, P, N), on-axis = 0 dB
    impedance: NDArray[np.complex128]                 # (F,) area-averaged pressure on the source tag
    observation_angles_deg: NDArray[np.float64]
    observation_points: NDArray[np.float64]
    observation_planes: list[str]
    config: SolveConfig
    mesh_info: MeshInfo
    timings: dict[str, float] = field(default_factory=dict)
    solver_log: list[dict] = field(default_factory=list)
    surface_pressure_avg: dict[int, NDArray[np.complex128]] | None = None
    surface_pressure_complex: NDArray[np.complex128] | None = None   # (F, n_p1)
    native_diagnostics: list[dict[str, Any]] = field(default_factory=list)

    @property
    def spl_norm_db(self) -> NDArray[np.float64]:
        return self.directivity_db
