"""Solve configuration for the B200 dense Helmholtz BEM path.

Field names, defaults and validation messages mirror the reference's
``SolveConfig`` / ``ObservationConfig`` (``hornlab_metal_bem/config.py:104-400``)
so a caller can swap packages without touching its configuration code.  The
``metal_native_*`` knobs are accepted for drop-in compatibility; on this
backend the threadgroup sizes map onto CUDA block-size overrides.

Three keys are new and only affect the B200 path:

* ``precision``: ``"plain"`` (FP32-accurate LU, the reference's complex64
  ``cgesv`` semantics) or ``"mixed"`` (BF16x3 tensor-core trailing updates).
  Either is followed by FP64-residual iterative refinement against the
  assembled matrix (the reference's optional refinement passes,
  ``main.swift:4855-4857, 6964-7070``).  Plain refines by default because an
  FP32 LU alone can lose digits to pivot growth: on the 1043-dof quarter horn
  at 16 kHz partial pivoting grows the entries ~8e3-fold and complex64
  ``cgesv`` (the reference's default) and this LU alike miss the FP64
  solution by 3e-3 to 5e-3, where one or two refinement passes recover 1e-6.
  ``refine_max_iterations=0`` keeps the unrefined cgesv result.
* ``refine_tolerance`` / ``refine_max_iterations``: refinement stopping rule:
  relative residual at most ``refine_tolerance``, at most
  ``refine_max_iterations`` passes, and a stop as soon as a pass no longer
  lowers the residual (the reference stops at 1e-7, after at most 10 passes
  or on the first pass that does not improve, ``main.swift:4995-5005``,
  ``6975-7063``).
* ``dense_solve_dtype="float64"`` (a reference key): the FP32-assembled
  system widened to complex128, factored and solved in FP64 on the GPU (the
  reference's ``zgesv`` path, ``main.swift:7101-7185``); no refinement.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from numbers import Integral
from typing import Any, Callable, Literal


class VelocityMode:
    VELOCITY = "velocity"
    ACCELERATION = "acceleration"


class SourceMotion:
    """How a driven tag's velocity maps onto its faces.

    ``NORMAL`` drives every face along its own outward normal at the same
    speed.  ``AXIAL`` drives a rigid piston along the frame axis, so each face
    gets ``U * (n_hat . axis)`` (``hornlab_metal_bem/config.py:18-33``).
    """

    NORMAL = "normal"
    AXIAL = "axial"


@dataclass(frozen=True)
class NormalProfile:
    """Uniform normal velocity on every face of the tag."""


@dataclass(frozen=True)
class AxialProfile:
    """Rigid piston: ``v_n = U * (n_hat . axis)``."""


@dataclass(frozen=True)
class TaperProfile:
    """Axial piston whose amplitude tapers to zero past ``start`` (normalised radius)."""

    kind: Literal["raised_cosine", "linear"] = "raised_cosine"
    start: float = 0.7


@dataclass(frozen=True)
class AnnularProfile:
    """Axial piston restricted to ``r_inner <= r/r_max <= r_outer``."""

    r_inner: float
    r_outer: float


@dataclass(frozen=True)
class PerFaceProfile:
    """Explicit per-face multipliers, in the tag's face order."""

    weights: object


@dataclass(frozen=True)
class CallableProfile:
    """``callback(centroids, unit_normals, axis, center) -> weights``."""

    callback: Callable[[object, object, object, object], object]


SourceProfile = (
    NormalProfile | AxialProfile | TaperProfile | AnnularProfile | PerFaceProfile | CallableProfile
)


class BIEFormulation:
    STANDARD = "standard"
    COMPLEX_K = "complex_k"


NATIVE_SYMMETRY_PLANES: tuple[str, ...] = ("yz", "xz", "xy", "yz+xz")

# Image-plane bit codes used across the C-ABI (reference ``main.swift:703-717``).
SYMMETRY_CODES: dict[str | None, int] = {None: 0, "yz": 1, "xz": 2, "yz+xz": 3, "xy": 4}


@dataclass
class ObservationConfig:
    planes: list[str] = field(default_factory=lambda: ["horizontal", "vertical"])
    distance_m: float = 2.0
    angle_min_deg: float = 0.0
    angle_max_deg: float = 180.0
    angle_count: int = 37
    origin: Literal["mouth", "throat"] = "mouth"
    custom_points: dict[str, Any] | None = None
    sphere_points: Any | None = None

    def __post_init__(self) -> None:
        if not self.planes:
            raise ValueError("observation planes must not be empty")
        if self.distance_m <= 0:
            raise ValueError("distance_m must be positive")
        if self.angle_count < 1:
            raise ValueError("angle_count must be at least 1")
        if self.origin not in ("mouth", "throat"):
            raise ValueError("origin must be 'mouth' or 'throat'")
        if self.sphere_points is not None:
            import numpy as np

            pts = np.asarray(self.sphere_points, dtype=float)
            if pts.ndim != 2 or pts.shape[1] != 3:
                raise ValueError("sphere_points must have shape (M, 3)")
            if pts.shape[0] == 0:
                raise ValueError("sphere_points must be non-empty when set")
            if not np.all(np.isfinite(pts)):
                raise ValueError("sphere_points must be finite")


def _positive_int_or_none(value: Any) -> bool:
    return value is None or (
        not isinstance(value, bool) and isinstance(value, Integral) and int(value) > 0
    )


@dataclass
class SolveConfig:
    freq_min_hz: float = 500.0
    freq_max_hz: float = 20_000.0
    freq_count: int = 40
    freq_spacing: Literal["log", "linear"] = "log"

    formulation: Literal["standard", "complex_k"] = BIEFormulation.STANDARD
    complex_k_shift: float = 0.005
    velocity_mode: Literal["velocity", "acceleration"] = VelocityMode.ACCELERATION
    source_motion: Literal["normal", "axial"] = SourceMotion.NORMAL
    source_velocity_profiles: dict[int, Any] | None = None
    velocity_sources: dict[int, complex] = field(default_factory=lambda: {2: 1.0})
    velocity_source_callback: Callable[[float], dict[int, complex]] | None = None
    impedance_sources: dict[int, complex] = field(default_factory=dict)
    impedance_source_callback: Callable[[float], dict[int, complex]] | None = None

    chief_points: Any | None = None
    chief_weight: float = 1.0

    circsym_baffle_z: float | None = None
    circsym_aperture_tag: int | None = None

    observation: ObservationConfig = field(default_factory=ObservationConfig)
    frame_override: object | None = None

    aperture_tag: int | None = None
    native_symmetry_plane: Literal["yz", "xz", "xy", "yz+xz"] | None = None
    native_check_open_edges: bool = True
    metal_native_assembly_mode: Literal["corrected", "optimized", "reference", "parity"] = "corrected"
    dense_solve_dtype: Literal["float32", "float64"] = "float32"
    return_surface_pressure: bool = False
    metal_native_threads_per_group: int | None = None
    metal_native_matrix_threads_per_group: int | None = None
    metal_native_rhs_threads_per_group: int | None = None
    metal_native_duffy_threads_per_group: int | None = None
    metal_native_field_threads_per_group: int | None = None

    dense_solve_rcond_warning_threshold: float = 1e-6
    mesh_elements_per_wavelength_min: float = 6.0

    mesh_scale: float = 1.0
    mesh_validate: bool = True
    mesh_merge_tol: float = 1e-9
    mesh_repair_normals: bool = False

    air_density: float = 1.2041

    progress_callback: Callable[[int, int, float], None] | None = None
    on_frequency_result: Callable[[int, float, dict], bool] | None = None

    # B200-only keys (no reference counterpart).
    precision: Literal["plain", "mixed"] = "plain"
    refine_tolerance: float = 1e-6
    refine_max_iterations: int = 10

    def __post_init__(self) -> None:
        if self.freq_spacing not in ("log", "linear"):
            raise ValueError("freq_spacing must be 'log' or 'linear'")
        if self.freq_count < 1:
            raise ValueError("freq_count must be at least 1")
        if self.freq_min_hz <= 0:
            raise ValueError("freq_min_hz must be positive")
        if self.freq_max_hz < self.freq_min_hz:
            raise ValueError("freq_max_hz must be >= freq_min_hz")
        if self.mesh_scale <= 0:
            raise ValueError("mesh_scale must be positive")
        if self.air_density <= 0:
            raise ValueError("air_density must be positive")
        if self.dense_solve_rcond_warning_threshold < 0:
            raise ValueError("dense_solve_rcond_warning_threshold must be non-negative")
        if self.mesh_elements_per_wavelength_min <= 0:
            raise ValueError("mesh_elements_per_wavelength_min must be positive")
        if self.formulation not in (BIEFormulation.STANDARD, BIEFormulation.COMPLEX_K):
            raise ValueError("formulation must be 'standard' or 'complex_k'")
        if self.complex_k_shift < 0:
            raise ValueError("complex_k_shift must be non-negative")
        if self.velocity_mode not in (VelocityMode.VELOCITY, VelocityMode.ACCELERATION):
            raise ValueError("velocity_mode must be 'velocity' or 'acceleration'")
        if self.source_motion not in (SourceMotion.NORMAL, SourceMotion.AXIAL):
            raise ValueError("source_motion must be 'normal' or 'axial'")
        if self.source_velocity_profiles is not None:
            if not isinstance(self.source_velocity_profiles, dict):
                raise ValueError("source_velocity_profiles must be a dict or None")
            for tag, profile in self.source_velocity_profiles.items():
                if int(tag) < 0:
                    raise ValueError("source_velocity_profiles tags must be non-negative integers")
                validate_source_profile(profile)
        for tag, beta in self.impedance_sources.items():
            if int(tag) < 0:
                raise ValueError("impedance_sources tags must be non-negative integers")
            value = complex(beta)
            if not (math.isfinite(value.real) and math.isfinite(value.imag)):
                raise ValueError("impedance_sources values must be finite complex numbers")
        if self.chief_points is not None:
            import numpy as np

            pts = np.asarray(self.chief_points, dtype=float)
            if pts.ndim != 2 or pts.shape[1] != 3:
                raise ValueError("chief_points must have shape (m, 3)")
            if pts.shape[0] == 0:
                raise ValueError("chief_points must be non-empty when set")
            if not np.all(np.isfinite(pts)):
                raise ValueError("chief_points must be finite")
        if not (math.isfinite(self.chief_weight) and self.chief_weight > 0):
            raise ValueError("chief_weight must be finite and positive")
        if self.circsym_baffle_z is not None and not math.isfinite(float(self.circsym_baffle_z)):
            raise ValueError("circsym_baffle_z must be finite or None")
        if not _positive_int_or_none(self.circsym_aperture_tag):
            raise ValueError("circsym_aperture_tag must be a positive int or None")
        if not _positive_int_or_none(self.aperture_tag):
            raise ValueError("aperture_tag must be a positive int or None")
        if (
            self.native_symmetry_plane is not None
            and self.native_symmetry_plane not in NATIVE_SYMMETRY_PLANES
        ):
            raise ValueError("native_symmetry_plane must be None, 'yz', 'xz', 'xy', or 'yz+xz'")
        if self.metal_native_assembly_mode not in ("corrected", "optimized", "reference", "parity"):
            raise ValueError(
                "metal_native_assembly_mode must be 'corrected', 'optimized', "
                "'reference', or 'parity'"
            )
        if self.dense_solve_dtype not in ("float32", "float64"):
            raise ValueError("dense_solve_dtype must be 'float32' or 'float64'")
        if self.metal_native_threads_per_group is not None and self.metal_native_threads_per_group <= 0:
            raise ValueError("metal_native_threads_per_group must be positive")
        for name in (
            "metal_native_matrix_threads_per_group",
            "metal_native_rhs_threads_per_group",
            "metal_native_duffy_threads_per_group",
            "metal_native_field_threads_per_group",
        ):
            value = getattr(self, name)
            if value is not None and value <= 0:
                raise ValueError(f"{name} must be positive")
        if self.precision not in ("plain", "mixed"):
            raise ValueError("precision must be 'plain' or 'mixed'")
        if not (self.refine_tolerance > 0 and math.isfinite(self.refine_tolerance)):
            raise ValueError("refine_tolerance must be finite and positive")
        if self.refine_max_iterations < 0:
            raise ValueError("refine_max_iterations must be non-negative")


def validate_source_profile(profile: Any) -> None:
    """Check one ``source_velocity_profiles`` value (``config.py:403-446`` of the reference)."""
    if isinstance(profile, (NormalProfile, AxialProfile)):
        return
    if isinstance(profile, TaperProfile):
        if profile.kind not in ("raised_cosine", "linear"):
            raise ValueError("TaperProfile.kind must be 'raised_cosine' or 'linear'")
        if not (math.isfinite(profile.start) and 0.0 <= profile.start < 1.0):
            raise ValueError("TaperProfile.start must be finite and in [0, 1)")
        return
    if isinstance(profile, AnnularProfile):
        ok = (
            math.isfinite(profile.r_inner)
            and math.isfinite(profile.r_outer)
            and 0.0 <= profile.r_inner <= profile.r_outer <= 1.0
        )
        if not ok:
            raise ValueError("AnnularProfile radii must be finite with 0 <= r_inner <= r_outer <= 1")
        return
    if isinstance(profile, PerFaceProfile):
        import numpy as np

        try:
            values = np.asarray(profile.weights, dtype=np.complex128)
        except (TypeError, ValueError) as exc:
            raise ValueError("PerFaceProfile.weights must be convertible to a complex array") from exc
        if values.ndim != 1 or values.size == 0:
            raise ValueError("PerFaceProfile.weights must be a non-empty 1D array")
        if not np.all(np.isfinite(values)):
            raise ValueError("PerFaceProfile.weights must be finite")
        return
    if isinstance(profile, CallableProfile):
        if not callable(profile.callback):
            raise ValueError("CallableProfile.callback must be callable")
        return
    raise ValueError("source_velocity_profiles values must be SourceProfile instances")
