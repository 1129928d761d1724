"""Boundary Lab backend adapter (the reference's ``hornlab_metal_bem/boundary_lab.py:133-935``).

Boundary Lab drives solvers through a small backend protocol: a backend object with an id and
capabilities, sessions created from a simulation config or a solve request, a one-shot ``solve`` and a
per-frequency ``solve_stream`` of ``FrequencyResult`` records.  This module translates Boundary Lab's
config fields into ``SolveConfig`` and the GPU sweep's per-frequency entries into those records.  It is
host code only: every solve goes through ``solve`` / ``solve_frequencies`` / ``solve_multi_source``.

Conventions kept from the reference: the BEM core is e^{-i omega t} (a source delayed by tau is
multiplied by e^{+i omega tau}; analog filter responses are the conjugates of scipy's e^{+j omega t}
ones), while Boundary Lab's channel synthesis uses the conjugate convention, so channel-basis pressures
and channel drives are conjugated once more before they are combined.
"""
from __future__ import annotations

import platform
import queue
import threading
from dataclasses import dataclass, field
from typing import Any, Callable, Iterable, Iterator

import numpy as np

from .config import BIEFormulation, ObservationConfig, SolveConfig, VelocityMode

REFERENCE_PRESSURE_PA = 20e-6
BACKEND_ID = "hornlab_metal"   # the id Boundary Lab configs name this backend by (drop-in)

try:  # Boundary Lab's own result types when it is installed
    from blab.solvers.base import (  # type: ignore[import-not-found]
        FrequencyResult,
        FrequencySolveTimings,
        SolveMetadata,
        SolverCapabilities,
        SolverDiagnostics,
    )
except Exception:  # standalone: the same record shapes
    @dataclass(frozen=True)
    class FrequencySolveTimings:
        assembly_s: float = 0.0
        solve_s: float = 0.0
        field_s: float = 0.0

    @dataclass(frozen=True)
    class SolverDiagnostics:
        convergence_info: int | None = None
        message: str | None = None

    @dataclass(frozen=True)
    class FrequencyResult:
        freq_hz: float
        horizontal_spl_norm_db: np.ndarray
        vertical_spl_norm_db: np.ndarray
        impedance: np.ndarray
        horizontal_spl_db: np.ndarray | None = None
        vertical_spl_db: np.ndarray | None = None
        sphere_spl_norm_db: np.ndarray | None = None
        channel_names: np.ndarray | None = None
        horizontal_pressure: np.ndarray | None = None
        vertical_pressure: np.ndarray | None = None
        sphere_pressure: np.ndarray | None = None
        timings: FrequencySolveTimings = field(default_factory=FrequencySolveTimings)
        diagnostics: SolverDiagnostics | None = None

        @property
        def has_channel_basis(self) -> bool:
            return all(x is not None for x in (self.channel_names, self.horizontal_pressure, self.vertical_pressure))

    @dataclass(frozen=True)
    class SolveMetadata:
        polar_angle_deg: np.ndarray
        radiator_names: np.ndarray
        sphere_metadata: dict[str, np.ndarray] | None = None

    @dataclass(frozen=True)
    class SolverCapabilities:
        supports_spherical_sampling: bool = False
        supports_impedance: bool = True
        supports_burton_miller: bool = False
        supports_flat_target_normalization: bool = True
        supports_channel_resynthesis: bool = True
        supports_cancellation: bool = True
        supports_streaming: bool = True
        supports_remote_assets: bool = False
        supports_parallel_workers: bool = False
        supports_symmetry: bool = True
        is_remote: bool = False


__all__ = [
    "BACKEND_ID",
    "BoundaryLabBackend",
    "BoundaryLabSession",
    "BoundaryLabSolverError",
    "create_backend",
    "is_apple_silicon",
    "is_cuda_available",
    "solve_config_from_boundary_lab",
]


class BoundaryLabSolverError(ValueError):
    pass


# --------------------------------------------------------------------------- field lookup
# Boundary Lab and hand-written specs spell several fields differently; the first name present wins.
_ALIASES: dict[str, tuple[str, ...]] = {
    "frequencies": ("frequencies_hz", "frequency_hz", "frequencies"),
    "planes": ("planes", "observation_planes"),
    "distance": ("distance", "distance_m", "observation_distance_m"),
    "origin": ("origin", "observation_origin"),
    "freq_min": ("freq_min", "freq_min_hz", "frequency_min_hz", "min_frequency_hz"),
    "freq_max": ("freq_max", "freq_max_hz", "frequency_max_hz", "max_frequency_hz"),
    "freq_count": ("freq_count", "frequency_count"),
    "freq_spacing": ("freq_spacing", "frequency_spacing"),
    "mesh_scale": ("mesh_scale", "scale_factor"),
    "air_density": ("rho", "air_density"),
    "check_open_edges": ("native_check_open_edges", "check_open_edges"),
    "angle_count": ("angle_count", "n_angles"),
    "angle_min": ("angle_min_deg", "min_angle_deg", "min_angle"),
    "angle_max": ("angle_max_deg", "max_angle_deg", "max_angle"),
    "angle_step": ("step_size", "polar_angle_step_deg"),
    "sphere_count": ("spherical_sampling_points", "balloon_sampling_points"),
    "axial_offset": ("axial_offset", "axial_offset_m"),
    "source_tag": ("source_tag", "driver_tag"),
    "source_weight": ("source_weight", "velocity_weight"),
}


def _field(source: Any, name: str, default: Any = None) -> Any:
    """Value of a field (alias list ``_ALIASES[name]``, else the name itself) of a dict or an object."""
    if source is None:
        return default
    for key in _ALIASES.get(name, (name,)):
        if isinstance(source, dict):
            if key in source:
                return source[key]
        elif hasattr(source, key):
            return getattr(source, key)
    return default


def _items(source: Any, name: str) -> tuple:
    return tuple(_field(source, name, ()) or ())


def _coerce_frequencies(value: Any) -> np.ndarray | None:
    if value is None:
        return None
    if isinstance(value, (int, float)):
        return np.array([float(value)])
    if isinstance(value, np.ndarray):
        return value.astype(np.float64)
    if isinstance(value, Iterable) and not isinstance(value, (str, bytes, dict)):
        return np.array([float(v) for v in value])
    raise BoundaryLabSolverError("frequencies_hz must be a number or sequence")


def _coerce_symmetry_plane(symmetry: Any) -> str | None:
    """Boundary Lab names the mirrored axes ("x": across X = 0, "xy": across X = 0 and Y = 0); the
    solver names the mirror planes ("yz" is X = 0, "xy" is Z = 0).  Plane names pass through."""
    token = str(symmetry or "off").strip().lower()
    mapped = {"": None, "off": None, "none": None, "x": "yz", "y": "xz", "z": "xy", "xy": "yz+xz",
              "yz": "yz", "xz": "xz", "yz+xz": "yz+xz"}
    if token not in mapped:
        raise BoundaryLabSolverError(f"Unsupported Boundary Lab symmetry mode: {symmetry!r}")
    return mapped[token]


# --------------------------------------------------------------------------- angles and sphere
def _boundary_lab_angles(source: Any) -> np.ndarray:
    """Polar angle grid: ``angle_count`` points over [min, max], else steps of ``step_size`` from min
    (the last step clipped to max, so the grid's last angle is the true end point)."""
    lo = float(_field(source, "angle_min", 0.0))
    hi = float(_field(source, "angle_max", 180.0))
    count = _field(source, "angle_count")
    if count is not None:
        return np.linspace(lo, hi, int(count))
    step = float(_field(source, "angle_step", 5.0))
    if step <= 0:
        raise BoundaryLabSolverError("step_size must be positive.")
    return np.minimum(np.arange(lo, hi + 0.5 * step, step), hi)


def _boundary_lab_sphere(source: Any):
    """Balloon sampling: a Fibonacci lattice of ``spherical_sampling_points`` points on the sphere of
    radius = observation distance about the origin (shifted by ``axial_offset`` along z), theta from
    +z, phi in the x-y plane.  Returns (points (N, 3), theta, phi, r) or None when disabled."""
    if not bool(_field(source, "spherical_sampling_enabled", False)):
        return None
    n = int(_field(source, "sphere_count", 6000))
    if n <= 0:
        return None
    radius = float(_field(source, "distance", 2.0))
    i = np.arange(n, dtype=np.float64)
    z = 1.0 - (2.0 * i + 1.0) / n
    phi = i * (np.pi * (3.0 - np.sqrt(5.0)))        # golden angle
    rho = np.sqrt(np.maximum(1.0 - z * z, 0.0))
    x, y = rho * np.cos(phi), rho * np.sin(phi)
    pts = radius * np.stack([x, y, z], axis=1)
    pts[:, 2] += float(_field(source, "axial_offset", 0.0))
    theta = np.arccos(np.clip(z, -1.0, 1.0)).astype(np.float32)
    azimuth = np.mod(np.arctan2(y, x), 2.0 * np.pi).astype(np.float32)
    return np.ascontiguousarray(pts), theta, azimuth, np.full(n, radius, dtype=np.float32)


# --------------------------------------------------------------------------- drives and filters
_CROSSOVER_KINDS = {"highpass": "highpass", "hpf": "highpass", "lowpass": "lowpass", "lpf": "lowpass"}


def _butterworth_response(kind: str, order: int, cutoff_hz: float, frequency_hz: float) -> complex:
    from scipy import signal

    b, a = signal.butter(order, 2.0 * np.pi * cutoff_hz, btype=kind, analog=True)
    _, h = signal.freqs(b, a, worN=[2.0 * np.pi * frequency_hz])
    return complex(np.conj(h[0]))                   # scipy's e^{+j w t} -> the core's e^{-i w t}


def _crossover_response(crossover: Any, frequency_hz: float) -> complex:
    """Analog Butterworth or Linkwitz-Riley (two cascaded Butterworth sections of half the order)
    high- or low-pass response at ``frequency_hz``, in the core's time convention."""
    kind = str(_field(crossover, "type", "none")).lower()
    if kind == "none":
        return 1.0 + 0.0j
    if kind not in _CROSSOVER_KINDS:
        raise BoundaryLabSolverError(f"Unsupported crossover type {kind!r}; expected one of "
                                     "'highpass', 'hpf', 'lowpass', 'lpf', or 'none'")
    family = str(_field(crossover, "filter", "butterworth")).lower()
    if family not in ("butterworth", "linkwitz_riley"):
        raise BoundaryLabSolverError(f"Unsupported crossover filter {family!r}; "
                                     "expected 'butterworth' or 'linkwitz_riley'")
    order = int(_field(crossover, "order", 1))
    if order < 1:
        raise BoundaryLabSolverError(f"crossover order must be >= 1, got {order}")
    cutoff = _field(crossover, "frequency_hz")
    if cutoff is None:
        raise BoundaryLabSolverError(f"crossover of type {kind!r} is missing frequency_hz")
    if float(cutoff) <= 0:
        raise BoundaryLabSolverError("crossover frequency_hz must be positive")
    if family == "linkwitz_riley":
        if order % 2:
            raise BoundaryLabSolverError(f"linkwitz_riley order must be even, got {order}")
        return _butterworth_response(_CROSSOVER_KINDS[kind], order // 2, float(cutoff), frequency_hz) ** 2
    return _butterworth_response(_CROSSOVER_KINDS[kind], order, float(cutoff), frequency_hz)


def _gain_polarity(source: Any) -> float:
    polarity = int(_field(source, "polarity", 1))
    if polarity not in (-1, 1):
        raise BoundaryLabSolverError(f"polarity must be -1 or 1, got {polarity!r}")
    return 10.0 ** (float(_field(source, "level_db", 0.0)) / 20.0) * polarity


def _filters(source: Any, frequency_hz: float) -> complex:
    h = 1.0 + 0.0j
    for name in ("hpf", "lpf"):
        cfg = _field(source, name)
        if cfg is not None and str(_field(cfg, "type", "none")).lower() != "none":
            h *= _crossover_response(cfg, frequency_hz)
    return h


def _level_polarity_delay_filter_drive(source: Any, frequency_hz: float) -> complex:
    """Source drive in the core's convention: level, polarity, delay tau as e^{+i omega tau}, filters."""
    omega = 2.0 * np.pi * float(frequency_hz)
    delay = np.exp(1j * omega * float(_field(source, "delay_ms", 0.0)) / 1000.0)
    return complex(_gain_polarity(source) * delay * _filters(source, frequency_hz))


def _boundary_lab_channel_drive(channel: Any, frequency_hz: float) -> complex:
    """Channel weight in Boundary Lab's synthesis convention: the conjugate of the core drive."""
    if channel is None:
        return 1.0 + 0.0j
    omega = 2.0 * np.pi * float(frequency_hz)
    delay = np.exp(-1j * omega * float(_field(channel, "delay_ms", 0.0)) / 1000.0)
    return complex(_gain_polarity(channel) * delay * np.conj(_filters(channel, frequency_hz)))


# --------------------------------------------------------------------------- sources and channels
def _offset_gain(radiator: Any) -> float:
    return 10.0 ** (float(_field(radiator, "velocity_offset_db", 0.0)) / 20.0)


def _coerce_velocity_sources(source: Any) -> dict[int, float]:
    explicit = _field(source, "velocity_sources")
    if explicit is not None:
        return {int(t): float(v) for t, v in dict(explicit).items()}
    radiators = _items(source, "radiators")
    if radiators:
        return {int(_field(r, "tag", 2)): 1.0 for r in radiators}
    return {int(_field(source, "source_tag", 2)): float(_field(source, "source_weight", 1.0))}


def _channel_configs_by_name(source: Any) -> dict[str, Any]:
    return {str(_field(c, "name", "main")): c for c in _items(source, "channels")}


def _boundary_lab_channel_configs_by_name(source: Any) -> dict[str, Any]:
    """Channel controls by name: the config's channels, else each channel's (last) radiator."""
    channels = _channel_configs_by_name(source)
    if channels:
        return channels
    return {str(_field(r, "channel", "main")): r for r in _items(source, "radiators")}


def _coerce_velocity_source_callback(source: Any) -> Callable[[float], dict[int, complex]] | None:
    """Per-frequency drives of radiator configs: each radiator's channel drive (or its own level,
    polarity, delay and filters without a channel) times its velocity offset, summed per tag."""
    if _field(source, "velocity_sources") is not None:
        return None
    radiators = _items(source, "radiators")
    if not radiators:
        return None
    channels = _channel_configs_by_name(source)

    def drives(frequency_hz: float) -> dict[int, complex]:
        out: dict[int, complex] = {}
        for r in radiators:
            tag = int(_field(r, "tag", 2))
            ch = channels.get(str(_field(r, "channel", "main")))
            d = _level_polarity_delay_filter_drive(r if ch is None else ch, frequency_hz) * _offset_gain(r)
            out[tag] = out.get(tag, 0.0 + 0.0j) + d
        return out

    return drives


def _channel_basis_sources(source: Any) -> tuple[np.ndarray, list[dict[int, complex]]]:
    """One unit source per channel (sorted channel names), radiator velocity offsets included;
    gain, polarity, delay and filters are applied after the solve by the channel synthesis."""
    radiators = _items(source, "radiators")
    if not radiators:
        return np.asarray(["main"]), [{t: complex(v) for t, v in _coerce_velocity_sources(source).items()}]
    names = sorted({str(_field(r, "channel", "main")) for r in radiators})
    basis = []
    for name in names:
        vec: dict[int, complex] = {}
        for r in radiators:
            if str(_field(r, "channel", "main")) == name:
                tag = int(_field(r, "tag", 2))
                vec[tag] = vec.get(tag, 0.0 + 0.0j) + complex(_offset_gain(r))
        basis.append(vec)
    return np.asarray(names), basis


def _radiator_names(source: Any) -> tuple[str, ...]:
    radiators = _items(source, "radiators")
    if not radiators:
        return ("throat",)
    return tuple(str(_field(r, "name", f"tag_{_field(r, 'tag', 2)}")) for r in radiators)


# --------------------------------------------------------------------------- config translation
def solve_config_from_boundary_lab(simulation_config: Any | None = None,
                                   **overrides: Any) -> tuple[SolveConfig, np.ndarray | None]:
    """``SolveConfig`` (and explicit frequencies, or None) from a Boundary Lab config given as a dict or
    an object; unknown fields are ignored, ``overrides`` replace translated values."""
    src = simulation_config
    angles = _boundary_lab_angles(src)
    sphere = _boundary_lab_sphere(src)
    observation = ObservationConfig(
        planes=list(_field(src, "planes", ["horizontal", "vertical"])),
        distance_m=float(_field(src, "distance", 2.0)),
        angle_min_deg=float(angles[0]),
        angle_max_deg=float(angles[-1]),
        angle_count=int(angles.size),
        origin=_field(src, "origin", "mouth"),
        sphere_points=None if sphere is None else sphere[0],
    )
    values: dict[str, Any] = dict(
        freq_min_hz=float(_field(src, "freq_min", 500.0)),
        freq_max_hz=float(_field(src, "freq_max", 20_000.0)),
        freq_count=int(_field(src, "freq_count", 40)),
        freq_spacing=_field(src, "freq_spacing", "log"),
        velocity_sources=_coerce_velocity_sources(src),
        velocity_source_callback=_coerce_velocity_source_callback(src),
        velocity_mode=VelocityMode.VELOCITY,
        # Boundary Lab's Burton-Miller switch asks for robustness at interior resonances; the complex
        # wavenumber formulation gives it here
        formulation=BIEFormulation.COMPLEX_K if bool(_field(src, "use_burton_miller", False))
        else BIEFormulation.STANDARD,
        mesh_scale=float(_field(src, "mesh_scale", 1.0)),
        air_density=float(_field(src, "air_density", 1.2041)),
        native_symmetry_plane=_coerce_symmetry_plane(_field(src, "symmetry", "off")),
        native_check_open_edges=bool(_field(src, "check_open_edges", True)),
        observation=observation,
        metal_native_assembly_mode="corrected",
    )
    values.update(overrides)
    return SolveConfig(**values), _coerce_frequencies(_field(src, "frequencies"))


# --------------------------------------------------------------------------- results
def _pressure_to_spl(p: np.ndarray) -> np.ndarray:
    with np.errstate(divide="ignore", invalid="ignore"):
        return (20.0 * np.log10(np.abs(p) / REFERENCE_PRESSURE_PA)).astype(np.float32)


def _plane_row(rows: np.ndarray, planes: list[str], plane: str, dtype) -> np.ndarray:
    if plane in planes:
        return np.asarray(rows[planes.index(plane)], dtype=dtype)
    return np.zeros(np.shape(rows)[-1], dtype=dtype)


def _impedance_pair(z: Any) -> np.ndarray:
    z = complex(0.0 if z is None else z)
    return np.array([z.real, z.imag], dtype=np.float32)


def _attach(result: Any, **extras: Any) -> None:
    for name, value in extras.items():
        try:
            object.__setattr__(result, name, value)
        except Exception:
            pass


def _timings(entries: list[dict[str, Any]]) -> FrequencySolveTimings:
    g = lambda e, *ks: next((float(e[k] or 0.0) for k in ks if k in e), 0.0)
    return FrequencySolveTimings(assembly_s=sum(g(e, "assembly_s") for e in entries),
                                 solve_s=sum(g(e, "dense_solve_s", "solve_s") for e in entries),
                                 field_s=sum(g(e, "field_s") for e in entries))


def _frequency_result_from_log_entry(frequency_hz: float, entry: dict[str, Any]) -> FrequencyResult:
    """One single-source streamed sweep entry as a ``FrequencyResult`` (normalised SPL from the
    sweep's directivity, raw SPL from the complex pressure when present)."""
    planes = list(entry.get("observation_planes") or ["horizontal", "vertical"])
    spl = np.asarray(entry["observation_directivity_db"], dtype=np.float32)
    p = entry.get("observation_pressure_complex")
    p = None if p is None else np.asarray(p, dtype=np.complex64)
    raw = (None, None) if p is None else tuple(_pressure_to_spl(_plane_row(p, planes, pl, np.complex64))
                                                for pl in ("horizontal", "vertical"))
    result = FrequencyResult(
        freq_hz=float(frequency_hz),
        horizontal_spl_norm_db=_plane_row(spl, planes, "horizontal", np.float32),
        vertical_spl_norm_db=_plane_row(spl, planes, "vertical", np.float32),
        impedance=_impedance_pair(entry.get("impedance"))[None, :],
        horizontal_spl_db=raw[0],
        vertical_spl_db=raw[1],
        sphere_spl_norm_db=None,
        timings=_timings([entry]),
        diagnostics=SolverDiagnostics(convergence_info=entry.get("lapack_info"),
                                      message=str(entry.get("backend", "native_metal"))),
    )
    _attach(result, observation_pressure_complex=p, native_diagnostics=dict(entry.get("native_diagnostics") or {}))
    return result


def _synthesize_boundary_lab_channel_basis(*, frequency_hz: float, channel_names: np.ndarray,
                                           channel_configs: dict[str, Any], horizontal_pressure: np.ndarray,
                                           vertical_pressure: np.ndarray, angles_deg: np.ndarray) -> dict:
    """Channel-weighted sum of the basis pressures, SPL re 20 uPa, normalised to the horizontal
    plane's value at the angle nearest 0 deg."""
    w = np.array([_boundary_lab_channel_drive(channel_configs.get(str(n)), frequency_hz)
                  for n in np.asarray(channel_names).tolist()], dtype=np.complex64)
    h = _pressure_to_spl(w @ horizontal_pressure)
    v = _pressure_to_spl(w @ vertical_pressure)
    ref = h[int(np.argmin(np.abs(angles_deg)))] if np.size(angles_deg) else h[0]
    return {"horizontal_spl_db": h, "vertical_spl_db": v,
            "horizontal_spl_norm_db": (h - ref).astype(np.float32), "vertical_spl_norm_db": (v - ref).astype(np.float32)}


def _frequency_result_from_channel_basis_entry(frequency_hz: float, entry: dict[str, Any], *,
                                               channel_names: np.ndarray,
                                               channel_configs: dict[str, Any]) -> FrequencyResult:
    """A multi-source streamed entry (``source_results``, one per channel; a plain entry is one channel)
    as a channel-basis ``FrequencyResult``: conjugated basis pressures per plane (and balloon),
    impedance per channel, and the channel synthesis at this frequency."""
    raw = entry.get("source_results")
    if raw is None:
        sources = [entry]
    elif isinstance(raw, list) and raw:
        sources = [dict(s) for s in raw]
    else:
        raise BoundaryLabSolverError("source_results must be a non-empty list.")
    names = np.asarray(channel_names)
    if len(sources) != names.size:
        raise BoundaryLabSolverError(f"Multi-source result count does not match the Boundary Lab channel count: "
                                     f"{len(sources)} result(s), {names.size} channel(s).")
    planes = list(entry.get("observation_planes") or ["horizontal", "vertical"])
    pressures = []
    for s in sources:
        if s.get("observation_pressure_complex") is None:
            raise BoundaryLabSolverError("The sweep result did not include observation_pressure_complex.")
        pressures.append(np.asarray(s["observation_pressure_complex"], dtype=np.complex64))
    hp = np.stack([np.conj(_plane_row(p, planes, "horizontal", np.complex64)) for p in pressures])
    vp = np.stack([np.conj(_plane_row(p, planes, "vertical", np.complex64)) for p in pressures])
    balloons = [s.get("observation_sphere_pressure_complex") for s in sources]
    sphere = (np.stack([np.conj(np.asarray(b, dtype=np.complex64)) for b in balloons])
              if all(b is not None for b in balloons) else None)
    angles = np.asarray(entry.get("observation_angles_deg", []), dtype=np.float32)
    if angles.size != hp.shape[1]:
        angles = np.linspace(0.0, 180.0, hp.shape[1], dtype=np.float32)
    syn = _synthesize_boundary_lab_channel_basis(frequency_hz=float(frequency_hz), channel_names=names,
                                                 channel_configs=channel_configs, horizontal_pressure=hp,
                                                 vertical_pressure=vp, angles_deg=angles)
    result = FrequencyResult(
        freq_hz=float(frequency_hz),
        horizontal_spl_norm_db=syn["horizontal_spl_norm_db"],
        vertical_spl_norm_db=syn["vertical_spl_norm_db"],
        impedance=np.stack([_impedance_pair(s.get("impedance")) for s in sources]),
        horizontal_spl_db=syn["horizontal_spl_db"],
        vertical_spl_db=syn["vertical_spl_db"],
        sphere_spl_norm_db=None,
        channel_names=names,
        horizontal_pressure=hp,
        vertical_pressure=vp,
        sphere_pressure=sphere,
        timings=_timings(sources),
        diagnostics=SolverDiagnostics(convergence_info=sources[0].get("lapack_info"),
                                      message=str(sources[0].get("backend", "native_metal"))),
    )
    _attach(result, observation_pressure_complex=np.stack(pressures),
            native_diagnostics=[dict(s.get("native_diagnostics") or {}) for s in sources])
    return result


# --------------------------------------------------------------------------- backend and sessions
def is_apple_silicon() -> bool:
    """The reference backend's platform test (kept for callers of that name)."""
    return platform.system() == "Darwin" and platform.machine() in {"arm64", "aarch64"}


def is_cuda_available() -> bool:
    """Whether this backend can run here: a CUDA device and the native library."""
    try:
        import torch

        if not torch.cuda.is_available():
            return False
        from .native import load_library

        load_library()
        return True
    except Exception:
        return False


@dataclass
class BoundaryLabSession:
    """A Boundary Lab solver session over the GPU sweep."""

    request_or_config: Any | None = None
    default_overrides: dict[str, Any] = field(default_factory=dict)
    _stop: bool = False

    @property
    def _simulation_config(self) -> Any | None:
        if self.request_or_config is None:
            return None
        nested = _field(self.request_or_config, "config")
        return self.request_or_config if nested is None else nested

    @property
    def _frequencies_hz(self) -> np.ndarray | None:
        return _coerce_frequencies(_field(self.request_or_config, "frequencies_hz"))

    @property
    def metadata(self) -> SolveMetadata:
        cfg = self._simulation_config
        sphere = _boundary_lab_sphere(cfg)
        return SolveMetadata(
            polar_angle_deg=_boundary_lab_angles(cfg).astype(np.float32),
            radiator_names=np.asarray(_radiator_names(cfg)),
            sphere_metadata=None if sphere is None else {
                "r_distance_m": sphere[3], "theta_polar_rad": sphere[1], "phi_azimuth_rad": sphere[2]},
        )

    def solve(self, mesh: Any, simulation_config: Any | None = None, **overrides: Any):
        """One ``SolveResult`` for the session's (or the given) config; request-level frequencies are used
        when the config has none."""
        from . import solve as _solve
        from . import solve_frequencies as _solve_frequencies

        cfg_source = self._simulation_config if simulation_config is None else simulation_config
        cfg, freqs = solve_config_from_boundary_lab(cfg_source, **{**self.default_overrides, **overrides})
        if freqs is None and simulation_config is None:
            freqs = self._frequencies_hz
        return _solve(mesh, cfg) if freqs is None else _solve_frequencies(mesh, freqs, cfg)

    def solve_stream(self, *, stop_requested: Callable[[], bool] | None = None) -> Iterator[FrequencyResult]:
        """Channel-basis ``FrequencyResult`` per frequency as the sweep completes them (one unit source per
        channel, solved on a worker thread); ``stop()`` or ``stop_requested()`` ends the sweep after the
        current frequency."""
        from . import solve_multi_source as _solve_multi_source

        self._stop = False    # a finished stream left it set; a new stream starts fresh
        cfg = self._simulation_config
        if cfg is None:
            raise BoundaryLabSolverError("Boundary Lab solve request is missing a SimulationConfig.")
        freqs = self._frequencies_hz
        if freqs is None:
            raise BoundaryLabSolverError("Boundary Lab solve request is missing frequencies_hz.")
        mesh_file = _field(cfg, "mesh_file")
        if mesh_file is None:
            raise BoundaryLabSolverError("Boundary Lab SimulationConfig is missing mesh_file.")
        names, basis = _channel_basis_sources(cfg)
        channel_configs = _boundary_lab_channel_configs_by_name(cfg)
        results: queue.Queue = queue.Queue()
        done = object()

        def stopping() -> bool:
            return self._stop or (stop_requested is not None and bool(stop_requested()))

        def on_frequency_result(index: int, frequency_hz: float, entry: dict[str, Any]) -> bool:
            results.put(_frequency_result_from_channel_basis_entry(frequency_hz, entry, channel_names=names,
                                                                   channel_configs=channel_configs))
            return not stopping()

        overrides = {**self.default_overrides, "on_frequency_result": on_frequency_result,
                     "velocity_sources": dict(basis[0]), "velocity_source_callback": None}
        solve_config, _ = solve_config_from_boundary_lab(cfg, **overrides)

        # a new host thread starts on CUDA device 0: run the sweep on the caller's current device
        device = _current_cuda_device()

        def work() -> None:
            try:
                if device is not None:
                    import torch

                    torch.cuda.set_device(device)
                _solve_multi_source(mesh_file, basis, solve_config, frequencies_hz=freqs)
            except BaseException as exc:   # re-raised in the consumer
                results.put(exc)
            finally:
                results.put(done)

        worker = threading.Thread(target=work, name="hornlab-b200-boundary-lab-solve", daemon=True)
        worker.start()
        try:
            while True:
                item = results.get()
                if item is done:
                    break
                if isinstance(item, BaseException):
                    raise item
                yield item
                if stopping():
                    self._stop = True
        finally:
            self._stop = True
            worker.join(timeout=1.0)

    def stop(self) -> None:
        self._stop = True

    def close(self) -> None:
        self.stop()

    def __enter__(self) -> "BoundaryLabSession":
        return self

    def __exit__(self, *exc: object) -> None:
        self.close()


@dataclass(frozen=True)
class BoundaryLabBackend:
    """Boundary Lab's local backend protocol for the B200 solver."""

    backend_id: str = BACKEND_ID
    label: str = "HornLab BEM (B200)"
    capabilities: SolverCapabilities = field(default_factory=lambda: SolverCapabilities(
        supports_spherical_sampling=True, supports_burton_miller=False, supports_flat_target_normalization=True,
        supports_channel_resynthesis=True, supports_cancellation=True, supports_streaming=True,
        supports_remote_assets=False, supports_parallel_workers=False, supports_symmetry=True, is_remote=False))
    default_overrides: dict[str, Any] = field(default_factory=dict)

    def create_session(self, request_or_config: Any | None = None) -> BoundaryLabSession:
        return BoundaryLabSession(request_or_config=request_or_config, default_overrides=dict(self.default_overrides))

    def supports(self, simulation_config: Any | None = None) -> bool:
        return is_cuda_available()


def create_backend(**default_overrides: Any) -> BoundaryLabBackend:
    return BoundaryLabBackend(default_overrides=dict(default_overrides))


def _current_cuda_device() -> int | None:
    """The calling thread's current CUDA device, or None without torch / CUDA."""
    try:
        import torch

        return int(torch.cuda.current_device()) if torch.cuda.is_available() else None
    except Exception:
        return None
