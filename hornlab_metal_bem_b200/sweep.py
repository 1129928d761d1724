"""Frequency sweep driver of the B200 path.

Mirrors ``hornlab_metal_bem/sweep.py`` of the reference: frequency grid
(``sweep.py:63-66``), float32 wavenumbers with the optional complex-k shift
(``:150-161``), per-frequency Neumann rows (``:238-285``), field points
(``:288-312``), directivity (``:523-532``), rcond / mesh-resolution policies
(``:383-440``) and ``SolveResult`` assembly (``:535-926``).  The solve itself
is one ``NativeSession.assemble_solve_evaluate_standard_neumann_batch`` call
per chunk of frequencies (all of them unless a streaming callback is set).
"""
from __future__ import annotations

import logging
import math
import time
from dataclasses import replace

import numpy as np

from ._constants import REFERENCE_PRESSURE, SPEED_OF_SOUND
from .bie import build_driver_neumann, build_source_face_scale
from .config import BIEFormulation, NATIVE_SYMMETRY_PLANES, SolveConfig
from .geometry import build_geometry_buffers
from .mesh import LoadedMesh, make_pure_function_spaces
from .native import BackendUnavailable, NativeSession
from .observation import ObservationFrame, build_observation_points
from .result import SolveResult

logger = logging.getLogger(__name__)


def build_frequency_grid(config: SolveConfig) -> np.ndarray:
    if config.freq_spacing == "log":
        return np.geomspace(config.freq_min_hz, config.freq_max_hz, config.freq_count)
    return np.linspace(config.freq_min_hz, config.freq_max_hz, config.freq_count)


def should_route_native(config: SolveConfig) -> bool:
    if config.native_symmetry_plane is not None and config.native_symmetry_plane not in NATIVE_SYMMETRY_PLANES:
        raise BackendUnavailable(
            "native_symmetry_plane must be None or one of " + ", ".join(repr(p) for p in NATIVE_SYMMETRY_PLANES)
        )
    if config.chief_points is not None and config.aperture_tag is not None:
        raise BackendUnavailable("chief_points with the coupled infinite baffle (aperture_tag): the coupled "
                                 "solve has no CHIEF rows")
    return True


def warn_near_boundary_chief_points(mesh: LoadedMesh, chief_points, max_edge_m: float) -> int:
    """Warn when CHIEF points sit within half the largest edge of the boundary (distance to the nearest
    vertex or triangle centroid): their constraint rows are exact only strictly inside the body, and a
    near-wall row biases the least squares with no error signal (the reference's check,
    ``sweep.py:342-380``).  Returns the number of such points."""
    vertices = np.asarray(mesh.grid.vertices, dtype=np.float64).T
    elements = np.asarray(mesh.grid.elements, dtype=np.int64).T
    if elements.size == 0 or max_edge_m <= 0.0:
        return 0
    anchors = np.vstack([vertices, vertices[elements].mean(axis=1)])
    pts = np.asarray(chief_points, dtype=np.float64).reshape(-1, 3)
    d2 = ((pts[:, None, :] - anchors[None, :, :]) ** 2).sum(axis=2)
    min_d = np.sqrt(d2.min(axis=1))
    near = np.nonzero(min_d < 0.5 * float(max_edge_m))[0]
    if near.size:
        worst = int(near[np.argmin(min_d[near])])
        logger.warning("%d of %d chief_points sit within 0.5*max_edge (%.4g m) of the boundary mesh (closest: "
                       "point %d at %.4g m); CHIEF points must be strictly interior", int(near.size),
                       int(pts.shape[0]), 0.5 * float(max_edge_m), worst, float(min_d[worst]))
    return int(near.size)


def impedance_sources_for_frequencies(physical_tags, frequencies, config: SolveConfig):
    """Robin admittance per frequency: the static ``impedance_sources`` dict, or one dict per
    frequency when ``impedance_source_callback`` is set (its values override / extend the static
    ones); tags absent from the mesh are skipped with a warning and non-passive values
    (``Re(beta) < 0``) or non-finite values from the callback raise (``sweep.py:164-239``)."""
    mesh_tags = {int(t) for t in np.unique(physical_tags)}
    static: dict[int, complex] = {}
    for tag, beta in (config.impedance_sources or {}).items():
        if int(tag) not in mesh_tags:
            logger.warning("impedance_sources references tag %d but mesh has no elements with that tag; skipping",
                           int(tag))
            continue
        static[int(tag)] = complex(beta)
    if config.impedance_source_callback is None:
        return [dict(static) for _ in np.atleast_1d(frequencies)]
    out = []
    for freq in np.atleast_1d(frequencies):
        f = float(freq)
        merged = dict(static)
        for tag, beta in config.impedance_source_callback(f).items():
            t = int(tag)
            if t not in mesh_tags:
                logger.warning("impedance_source_callback returned tag %d not in mesh; skipping", t)
                continue
            b = complex(beta)
            if not (math.isfinite(b.real) and math.isfinite(b.imag)):
                raise ValueError(f"impedance_source_callback({f:.3f}) returned non-finite beta for tag {t}")
            if b.real < 0.0:
                raise ValueError(f"impedance_source_callback({f:.3f}) returned Re(beta)={b.real:.4g} < 0 for tag {t}; "
                                 "admittance must be passive (Re(beta) >= 0)")
            merged[t] = b
        out.append(merged)
    return out


def k_values(frequencies, config: SolveConfig) -> tuple[np.ndarray, np.ndarray]:
    """``k = float32(2 pi f / c)``; complex-k adds ``i * shift * k`` (``sweep.py:150-161``)."""
    k_re = (2.0 * np.pi * np.asarray(frequencies, dtype=np.float64) / SPEED_OF_SOUND).astype(np.float32)
    if config.formulation == BIEFormulation.COMPLEX_K:
        k_im = (k_re.astype(np.float64) * config.complex_k_shift).astype(np.float32)
    else:
        k_im = np.zeros_like(k_re)
    return k_re, k_im


def neumann_rows(n_faces: int, physical_tags, frequencies, config: SolveConfig, source_face_scale=None,
                 impedance_per_freq=None) -> np.ndarray:
    """Driver Neumann rows; Robin tags of each frequency are skipped as velocity sources (``sweep.py:242-285``)."""
    rows = []
    for i, f in enumerate(frequencies):
        tags_robin = (set(impedance_per_freq[i].keys()) if impedance_per_freq is not None
                      else set(config.impedance_sources.keys()))
        rows.append(build_driver_neumann(n_faces, physical_tags, 2.0 * np.pi * float(f), config, np.complex64,
                                         impedance_tags=tags_robin, source_face_scale=source_face_scale))
    return np.stack(rows)


def field_points_3xn(obs_points: np.ndarray) -> np.ndarray:
    p, n, _ = obs_points.shape
    return np.ascontiguousarray(obs_points.reshape(p * n, 3).T, dtype=np.float32)


def directivity_from_pressure(pressure: np.ndarray, on_axis_idx: int) -> np.ndarray:
    """SPL re 20 uPa, floored at -120 dB SPL, minus the on-axis value per plane."""
    floor = REFERENCE_PRESSURE * 10.0 ** (-120.0 / 20.0)
    spl = 20.0 * np.log10(np.maximum(np.abs(pressure), floor) / REFERENCE_PRESSURE)
    return spl - spl[:, on_axis_idx][:, None]


def mesh_max_edge(mesh: LoadedMesh) -> float:
    v = np.asarray(mesh.grid.vertices, dtype=np.float64).T
    f = np.asarray(mesh.grid.elements).T
    if f.size == 0:
        return 0.0
    e = [np.linalg.norm(v[f[:, (i + 1) % 3]] - v[f[:, i]], axis=1).max() for i in range(3)]
    return float(max(e))


def apply_dense_solve_policy(diag: dict, threshold: float) -> None:
    diag["dense_solve_rcond_warning_threshold"] = float(threshold)
    diag["dense_solve_suspect"] = False
    if threshold <= 0.0:
        return
    rcond = diag.get("dense_solve_rcond")
    if rcond is None:
        diag["dense_solve_policy_available"] = False
        return
    diag["dense_solve_policy_available"] = True
    if math.isfinite(float(rcond)) and float(rcond) < threshold:
        diag["dense_solve_suspect"] = True
        diag["dense_solve_recommendation"] = (
            "Treat this frequency as suspect; nudge or densify the frequency grid around the resonance "
            "and compare against nearby points. This flag detects dense-solve conditioning only."
        )


def apply_mesh_resolution_policy(diag: dict, frequency_hz: float, max_edge: float, epw_min: float) -> None:
    diag["mesh_max_edge_m"] = float(max_edge)
    diag["mesh_elements_per_wavelength_min"] = float(epw_min)
    if max_edge <= 0.0:
        diag["mesh_elements_per_wavelength"] = math.inf
        diag["mesh_max_valid_frequency_hz"] = math.inf
        diag["mesh_resolution_suspect"] = False
        return
    epw = (SPEED_OF_SOUND / float(frequency_hz)) / max_edge
    diag["mesh_elements_per_wavelength"] = float(epw)
    diag["mesh_max_valid_frequency_hz"] = float(SPEED_OF_SOUND / (epw_min * max_edge))
    diag["mesh_resolution_suspect"] = bool(epw < epw_min)


def run_sweep(mesh: LoadedMesh, frequencies, frame: ObservationFrame, config: SolveConfig,
              *, session: NativeSession | None = None, average_tags=None) -> SolveResult:
    """Standard-Neumann sweep on the GPU (the reference's ``run_sweep_native_metal``).

    ``average_tags`` adds tags to the surface-pressure averages (the sorted union with the
    velocity-source tags is recorded); multi-source sweeps pass every source's tags."""
    return _run_sweep_sources(mesh, frequencies, frame, [config], session=session, average_tags=average_tags)[0]


def _run_sweep_sources(mesh: LoadedMesh, frequencies, frame: ObservationFrame, configs: list[SolveConfig],
                       *, session: NativeSession | None = None, average_tags=None) -> list[SolveResult]:
    """One sweep for one or more velocity-source configurations that differ only in their sources.

    With several sources every frequency's matrix is assembled and factored once and each source is a
    right-hand side of it (the reference's multi-RHS sweep, ``sweep.py:957-1301`` with
    ``main.swift:6348-6368, 7887``); the streaming callback then fires once per frequency with the first
    source's entry plus ``source_results`` (one entry per source)."""
    config = configs[0]
    for c in configs:
        should_route_native(c)
    freqs = np.asarray(frequencies, dtype=np.float64)
    if freqs.size == 0:
        raise ValueError("frequencies must contain at least one value")
    mesh_tags = {int(t) for t in np.unique(mesh.physical_tags)}
    for c in configs:
        missing = sorted(set(c.velocity_sources) - mesh_tags)
        if missing:
            raise ValueError(
                f"velocity_sources tags {missing} are not present in the mesh; available physical tags: "
                f"{sorted(mesh_tags)}"
            )
    n_src = len(configs)
    t_total = time.time()
    obs_points, angles = build_observation_points(frame, config.observation)
    p1, dp0 = make_pure_function_spaces(mesh.grid)
    buffers = build_geometry_buffers(mesh.grid, mesh.physical_tags, p1, dp0)
    max_edge = mesh_max_edge(mesh)
    source_tags = sorted({int(t) for c in configs for t in c.velocity_sources})
    if n_src == 1:
        source_tags = list(config.velocity_sources.keys())
    if average_tags is not None:
        source_tags = sorted({int(t) for t in source_tags} | {int(t) for t in average_tags})
    on_axis = int(np.argmin(np.abs(angles)))
    imp_tags = [min(c.velocity_sources.keys(), default=2) for c in configs]
    n_planes, n_angles, _ = obs_points.shape
    pts = field_points_3xn(obs_points)
    n_sphere = 0
    if config.observation.sphere_points is not None:
        sp = np.ascontiguousarray(np.asarray(config.observation.sphere_points, dtype=np.float64).T, dtype=np.float32)
        n_sphere = sp.shape[1]
        pts = np.concatenate([pts, sp], axis=1)
    k_re, k_im = k_values(freqs, config)
    robin = None
    if config.impedance_sources or config.impedance_source_callback is not None:
        robin = impedance_sources_for_frequencies(mesh.physical_tags, freqs, config)
        if not any(robin):
            robin = None
    if n_src > 1 and (robin is not None or config.aperture_tag is not None):
        raise ValueError("shared-factorisation multi-source sweeps support neither Robin walls nor the coupled baffle")
    qs = []
    for c in configs:
        scale = build_source_face_scale(mesh.grid, mesh.physical_tags, c, frame.axis, frame.source_center)
        qs.append(neumann_rows(buffers.n_triangles, mesh.physical_tags, freqs, c, scale, robin))
    q = qs[0]
    extra = np.stack(qs[1:], axis=0) if n_src > 1 else None
    chief = None
    if config.chief_points is not None:
        chief = np.ascontiguousarray(np.asarray(config.chief_points, dtype=np.float64).T, dtype=np.float32)
        warn_near_boundary_chief_points(mesh, config.chief_points, max_edge)

    own = session is None
    if own:
        session = NativeSession(buffers, symmetry_plane=config.native_symmetry_plane,
                                aperture_tag=config.aperture_tag, velocity_source_tags=source_tags,
                                check_open_edges=config.native_check_open_edges)
    rows = [dict(pressure=[], spl=[], imp=[], surf=[], diag=[], log=[], pavg={t: [] for t in source_tags})
            for _ in configs]
    done: list[float] = []
    try:
        chunk = freqs.size if config.on_frequency_result is None else 1
        stop = False
        for f0 in range(0, freqs.size, chunk):
            sl = slice(f0, f0 + chunk)
            batch_fn = (session.coupled_ib_batch if config.aperture_tag is not None
                        else session.assemble_solve_evaluate_standard_neumann_batch)
            kw = {}
            if extra is not None:
                kw = dict(extra_neumann_dp0=extra[:, sl], extra_impedance_source_tags=imp_tags[1:])
            if chief is not None:
                kw.update(chief_points=chief, chief_weight=config.chief_weight)
            results = batch_fn(
                freqs[sl], k_re[sl], q[sl], pts, k_imag_f32=k_im[sl], source_tags=source_tags,
                impedance_source_tag=imp_tags[0], write_surface_pressure=config.return_surface_pressure,
                dense_solve_dtype=config.dense_solve_dtype, precision=config.precision,
                refine_tolerance=config.refine_tolerance, refine_max_iterations=config.refine_max_iterations,
                compute_rcond=config.dense_solve_rcond_warning_threshold > 0,
                impedance_sources=None if robin is None else robin[sl], **kw,
            )
            for j, res in enumerate(results):
                i = f0 + j
                if res.lapack_info != 0:
                    raise RuntimeError(f"dense LU failed at {res.frequency_hz:.3f} Hz: zero pivot {res.lapack_info}")
                diag0 = dict(res.diagnostics)
                apply_dense_solve_policy(diag0, config.dense_solve_rcond_warning_threshold)
                apply_mesh_resolution_policy(diag0, res.frequency_hz, max_edge, config.mesh_elements_per_wavelength_min)
                entries = []
                for s_, acc in enumerate(rows):
                    out = res if s_ == 0 else res.extra_sources[s_ - 1]
                    flat = out.field.astype(np.complex128)
                    arc = flat[: n_planes * n_angles].reshape(n_planes, n_angles)
                    sphere = flat[n_planes * n_angles:] if n_sphere else None
                    spl = directivity_from_pressure(arc, on_axis)
                    diag = dict(diag0)
                    if s_ > 0:
                        diag.update(refine_iterations=out.refine_iterations,
                                    refine_residual_rel=out.refine_residual_rel, source_index=s_)
                    for t in source_tags:
                        acc["pavg"][t].append(out.surface_pressure_avg[int(t)])
                    entry = {
                        "frequency_hz": res.frequency_hz,
                        "iterations": None,
                        "timing_s": res.assembly_s + res.dense_solve_s + res.field_s,
                        "backend": "hbem_b200_batch" if chunk > 1 else "hbem_b200_streamed",
                        "assembly_s": res.assembly_s,
                        "dense_solve_s": res.dense_solve_s,
                        "field_s": res.field_s,
                        "lapack_info": res.lapack_info,
                        "impedance": out.impedance,
                        "native_diagnostics": diag,
                        "observation_sphere_pressure_complex": sphere,
                    }
                    acc["pressure"].append(arc)
                    acc["spl"].append(spl)
                    acc["imp"].append(out.impedance)
                    if config.return_surface_pressure:
                        acc["surf"].append(out.surface_pressure.astype(np.complex128))
                    acc["diag"].append(diag)
                    acc["log"].append(entry)
                    entries.append({**entry, "observation_pressure_complex": arc, "observation_directivity_db": spl,
                                    "observation_angles_deg": angles,
                                    "observation_planes": config.observation.planes})
                done.append(res.frequency_hz)
                if config.progress_callback is not None:
                    config.progress_callback(i, freqs.size, res.frequency_hz)
                if config.on_frequency_result is not None:
                    cb = entries[0] if n_src == 1 else {**entries[0], "source_results": entries}
                    if config.on_frequency_result(i, res.frequency_hz, cb) is False:
                        logger.info("Early stop requested after %.1f Hz", res.frequency_hz)
                        stop = True
                        break
            if stop:
                break
    finally:
        if own:
            session.close()
    out_results = []
    for c, acc in zip(configs, rows):
        log = acc["log"]
        timings = {
            "solve_s": sum(e["timing_s"] for e in log),
            "assembly_s": sum(e["assembly_s"] for e in log),
            "dense_solve_s": sum(e["dense_solve_s"] for e in log),
            "directivity_s": sum(e["field_s"] for e in log),
            "total_s": time.time() - t_total,
        }
        out_results.append(SolveResult(
            frequencies_hz=np.array(done, dtype=np.float64),
            pressure_complex=np.stack(acc["pressure"], axis=0),
            directivity_db=np.stack(acc["spl"], axis=0),
            impedance=np.array(acc["imp"], dtype=np.complex128),
            observation_angles_deg=angles,
            observation_points=obs_points,
            observation_planes=config.observation.planes,
            config=c,
            mesh_info=mesh.info,
            timings=timings,
            solver_log=log,
            surface_pressure_avg={t: np.array(v, dtype=np.complex128) for t, v in acc["pavg"].items()} or None,
            surface_pressure_complex=np.stack(acc["surf"], axis=0) if config.return_surface_pressure else None,
            native_diagnostics=acc["diag"],
        ))
    return out_results


def run_sweep_multi_source(mesh: LoadedMesh, frequencies, frame: ObservationFrame, config: SolveConfig,
                           sources: list[dict[int, complex]]) -> list[SolveResult]:
    """One result per velocity-source dict (the reference's ``run_sweep_native_metal_multi_source``,
    ``sweep.py:957-1301``), every source on one resident session, each result recording the surface
    averages of the sorted union of all source tags.

    Every frequency's matrix is assembled and factored once for all sources: one assembly pass fills the
    matrix and each source's right-hand side, one LU, one solve per source (the reference's multi-RHS
    ``cgesv``, ``main.swift:7887``).  With ``on_frequency_result`` the callback runs once per frequency with
    the first source's entry plus ``source_results`` (one entry per source), as the reference's multi-RHS
    stream; returning False stops after that frequency and the results hold the completed frequencies.
    Robin walls and the coupled baffle solve one source at a time (same results, one factorisation per
    source).  ``velocity_source_callback`` is rejected: each source vector is fixed for the whole sweep.
    """
    if not sources:
        raise ValueError("sources must contain at least one velocity dict")
    if config.velocity_source_callback is not None:
        raise ValueError("multi-source solves do not support velocity_source_callback")
    p1, dp0 = make_pure_function_spaces(mesh.grid)
    buffers = build_geometry_buffers(mesh.grid, mesh.physical_tags, p1, dp0)
    all_tags = sorted({int(t) for s in sources for t in s})
    per_source = [replace(config, velocity_sources=dict(src)) for src in sources]
    shared = not (config.impedance_sources or config.impedance_source_callback is not None
                  or config.aperture_tag is not None)
    with NativeSession(buffers, symmetry_plane=config.native_symmetry_plane, aperture_tag=config.aperture_tag,
                       velocity_source_tags=all_tags, check_open_edges=config.native_check_open_edges) as session:
        if shared:
            return _run_sweep_sources(mesh, frequencies, frame, per_source, session=session, average_tags=all_tags)
        if config.on_frequency_result is None:
            return [run_sweep(mesh, frequencies, frame, c, session=session, average_tags=all_tags)
                    for c in per_source]
        quiet = [replace(c, on_frequency_result=None, progress_callback=None) for c in per_source]
        freqs = np.atleast_1d(np.asarray(frequencies, dtype=np.float64))
        parts: list[list[SolveResult]] = [[] for _ in sources]
        for i, f in enumerate(freqs):
            entries = []
            for s, c in enumerate(quiet):
                r = run_sweep(mesh, [f], frame, c, session=session, average_tags=all_tags)
                parts[s].append(r)
                entry = dict(r.solver_log[-1])
                entry.update(observation_pressure_complex=r.pressure_complex[0],
                             observation_directivity_db=r.directivity_db[0],
                             observation_angles_deg=r.observation_angles_deg,
                             observation_planes=r.observation_planes)
                entries.append(entry)
            if config.progress_callback is not None:
                config.progress_callback(i, freqs.size, float(f))
            if config.on_frequency_result(i, float(f), {**entries[0], "source_results": entries}) is False:
                logger.info("Early stop requested after %.1f Hz", float(f))
                break
        return [_concat_results(p, c) for p, c in zip(parts, per_source)]


def _concat_results(parts: list[SolveResult], config: SolveConfig) -> SolveResult:
    """One ``SolveResult`` from per-frequency results of the same source, in order."""
    first = parts[0]
    cat = lambda name: np.concatenate([getattr(p, name) for p in parts], axis=0)
    return SolveResult(
        frequencies_hz=cat("frequencies_hz"),
        pressure_complex=cat("pressure_complex"),
        directivity_db=cat("directivity_db"),
        impedance=cat("impedance"),
        observation_angles_deg=first.observation_angles_deg,
        observation_points=first.observation_points,
        observation_planes=first.observation_planes,
        config=config,
        mesh_info=first.mesh_info,
        timings={k: sum(float(p.timings.get(k, 0.0)) for p in parts) for k in first.timings},
        solver_log=[e for p in parts for e in p.solver_log],
        surface_pressure_avg=None if first.surface_pressure_avg is None else {
            t: np.concatenate([p.surface_pressure_avg[t] for p in parts]) for t in first.surface_pressure_avg},
        surface_pressure_complex=None if first.surface_pressure_complex is None else cat("surface_pressure_complex"),
        native_diagnostics=[d for p in parts for d in p.native_diagnostics],
    )
