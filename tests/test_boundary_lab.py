"""Boundary Lab backend adapter (host only): config translation, request handling, metadata, sphere
sampling, drives and crossovers, symmetry tokens, result records and the channel-basis stream, as the
reference's tests pin them (tests/test_boundary_lab_backend.py:17-430).  Solves are replaced by fakes."""
from __future__ import annotations

from types import SimpleNamespace

import numpy as np
import pytest

from hornlab_metal_bem_b200.boundary_lab import (
    BACKEND_ID,
    BoundaryLabSolverError,
    _coerce_symmetry_plane,
    _crossover_response,
    _frequency_result_from_channel_basis_entry,
    _frequency_result_from_log_entry,
    _level_polarity_delay_filter_drive,
    create_backend,
    solve_config_from_boundary_lab,
)


def test_config_translation_defaults_and_aliases():
    cfg, freqs = solve_config_from_boundary_lab({"frequency_min_hz": 800.0, "frequency_max_hz": 12_500.0,
                                                 "frequency_count": 9, "source_tag": 7,
                                                 "observation_planes": ["horizontal"]})
    assert freqs is None
    assert (cfg.freq_min_hz, cfg.freq_max_hz, cfg.freq_count) == (800.0, 12_500.0, 9)
    assert cfg.velocity_sources == {7: 1.0} and cfg.observation.planes == ["horizontal"]
    assert cfg.velocity_mode == "velocity" and cfg.metal_native_assembly_mode == "corrected"
    assert solve_config_from_boundary_lab({"symmetry": "yz+xz"})[0].native_check_open_edges is True
    assert solve_config_from_boundary_lab({"symmetry": "yz+xz", "native_check_open_edges": False})[0] \
        .native_check_open_edges is False
    assert solve_config_from_boundary_lab({"symmetry": "yz+xz", "check_open_edges": False})[0] \
        .native_check_open_edges is False
    src = SimpleNamespace(frequencies_hz=[1000.0, 1600.0], velocity_sources={3: 0.5}, angle_count=5)
    cfg, freqs = solve_config_from_boundary_lab(src, metal_native_threads_per_group=64)
    np.testing.assert_allclose(freqs, [1000.0, 1600.0])
    assert cfg.velocity_sources == {3: 0.5} and cfg.observation.angle_count == 5
    assert cfg.metal_native_threads_per_group == 64
    for flag, want in ((True, "complex_k"), (False, "standard")):
        assert solve_config_from_boundary_lab({"use_burton_miller": flag})[0].formulation == want
    assert solve_config_from_boundary_lab({})[0].formulation == "standard"


def test_backend_sessions_and_requests():
    backend = create_backend(freq_count=3)
    session = backend.create_session({"freq_min_hz": 900.0})
    assert backend.backend_id == BACKEND_ID and backend.capabilities.supports_channel_resynthesis is True
    assert session.default_overrides == {"freq_count": 3}
    s = create_backend().create_session({"config": {"frequency_count": 7, "source_tag": 3},
                                         "frequencies_hz": [100.0, 200.0]})
    assert s._simulation_config == {"frequency_count": 7, "source_tag": 3}
    np.testing.assert_allclose(s._frequencies_hz, [100.0, 200.0])
    config = SimpleNamespace(mesh_file="waveguide.msh", min_angle=-90.0, max_angle=90.0, step_size=45.0,
                             radiators=(SimpleNamespace(name="Woofer", tag=7, velocity_offset_db=6.0),))
    s = create_backend().create_session(SimpleNamespace(config=config, frequencies_hz=np.array([1e3, 1.6e3])))
    assert s.metadata.polar_angle_deg.tolist() == [-90.0, -45.0, 0.0, 45.0, 90.0]
    assert s.metadata.radiator_names.tolist() == ["Woofer"]
    cfg, freqs = solve_config_from_boundary_lab(config)
    assert freqs is None and cfg.velocity_sources[7] == 1.0
    assert cfg.velocity_source_callback(1000.0)[7] == pytest.approx(10.0 ** (6.0 / 20.0))
    assert (cfg.observation.angle_min_deg, cfg.observation.angle_max_deg, cfg.observation.angle_count) == (-90, 90, 5)


def test_angle_grid_with_a_step_that_does_not_divide_the_span():
    config = {"min_angle": 0.0, "max_angle": 100.0, "step_size": 30.0}
    meta = create_backend().create_session({"config": config}).metadata
    cfg, _ = solve_config_from_boundary_lab(config)
    solved = np.linspace(cfg.observation.angle_min_deg, cfg.observation.angle_max_deg, cfg.observation.angle_count)
    np.testing.assert_allclose(meta.polar_angle_deg, solved)
    np.testing.assert_allclose(solved, [0.0, 30.0, 60.0, 90.0])
    with pytest.raises(BoundaryLabSolverError, match="step_size"):
        solve_config_from_boundary_lab({"step_size": 0.0})


def test_spherical_sampling():
    config = {"mesh_file": "m.msh", "spherical_sampling_enabled": True, "spherical_sampling_points": 32,
              "distance": 3.0}
    cfg, _ = solve_config_from_boundary_lab(config)
    pts = cfg.observation.sphere_points
    assert pts.shape == (32, 3)
    np.testing.assert_allclose(np.linalg.norm(pts, axis=1), 3.0, atol=1e-5)
    assert abs(pts.mean(axis=0)).max() < 0.2           # a balanced lattice over the sphere
    meta = create_backend().create_session({"config": config}).metadata
    assert set(meta.sphere_metadata) == {"r_distance_m", "theta_polar_rad", "phi_azimuth_rad"}
    assert meta.sphere_metadata["theta_polar_rad"].shape == (32,)
    assert solve_config_from_boundary_lab({"mesh_file": "m.msh"})[0].observation.sphere_points is None
    assert create_backend().create_session({"config": {"mesh_file": "m.msh"}}).metadata.sphere_metadata is None


def test_drives_and_crossovers():
    # e^{-i omega t}: a 1 ms delay at 250 Hz is a quarter turn forward, 1 -> +i
    np.testing.assert_allclose(_level_polarity_delay_filter_drive({"delay_ms": 1.0}, 250.0), 1j, atol=1e-12)
    assert _level_polarity_delay_filter_drive({"level_db": 6.0, "polarity": -1}, 1e3) == \
        pytest.approx(-(10.0 ** 0.3))
    with pytest.raises(BoundaryLabSolverError, match="polarity"):
        _level_polarity_delay_filter_drive({"polarity": 0}, 1000.0)
    # first-order Butterworth low-pass at its cutoff: 1/(1+j) for scipy, so 1/(1-j) here
    lp = _crossover_response({"type": "lpf", "filter": "butterworth", "order": 1, "frequency_hz": 1000.0}, 1000.0)
    np.testing.assert_allclose(lp, 1.0 / (1.0 - 1.0j), rtol=1e-9)
    lr4 = _crossover_response({"type": "lpf", "filter": "linkwitz_riley", "order": 4, "frequency_hz": 1e3}, 1e3)
    np.testing.assert_allclose(abs(lr4), 0.5, rtol=1e-9)       # LR4: -6 dB at the cutoff
    assert _crossover_response({"type": "none"}, 1e3) == 1.0


@pytest.mark.parametrize(("crossover", "match"), [
    ({"type": "bandpass", "frequency_hz": 1000.0}, "crossover type"),
    ({"type": "lpf", "filter": "bessel", "frequency_hz": 1000.0}, "crossover filter"),
    ({"type": "lpf"}, "missing frequency_hz"),
    ({"type": "lpf", "frequency_hz": 0.0}, "must be positive"),
    ({"type": "lpf", "order": 0, "frequency_hz": 1000.0}, "order"),
    ({"type": "lpf", "filter": "linkwitz_riley", "order": 3, "frequency_hz": 1000.0}, "even"),
])
def test_crossover_rejections(crossover, match):
    with pytest.raises(BoundaryLabSolverError, match=match):
        _crossover_response(crossover, 2000.0)


@pytest.mark.parametrize(("token", "plane"), [("off", None), ("x", "yz"), ("y", "xz"), ("z", "xy"),
                                              ("xy", "yz+xz"), ("yz", "yz"), ("xz", "xz"), ("yz+xz", "yz+xz")])
def test_symmetry_tokens(token, plane):
    assert _coerce_symmetry_plane(token) == plane


def test_symmetry_token_rejected():
    with pytest.raises(BoundaryLabSolverError, match="symmetry"):
        _coerce_symmetry_plane("diagonal")


def test_log_entry_result_keeps_the_streamed_pressure():
    p = np.array([[1.0 + 1.0j, 2.0 - 1.0j], [0.5 + 0.25j, 0.25 - 0.5j]])
    r = _frequency_result_from_log_entry(1000.0, {
        "observation_planes": ["horizontal", "vertical"], "observation_directivity_db": np.zeros((2, 2)),
        "observation_pressure_complex": p, "impedance": 1.0 + 0.5j, "lapack_info": 0,
        "native_diagnostics": {"assembly_implementation": "test"}})
    np.testing.assert_allclose(r.observation_pressure_complex, p, rtol=1e-6)
    np.testing.assert_allclose(r.horizontal_spl_db, 20.0 * np.log10(np.abs(p[0]) / 20e-6), rtol=1e-5)
    assert r.native_diagnostics["assembly_implementation"] == "test" and r.diagnostics.convergence_info == 0
    np.testing.assert_allclose(r.impedance, [[1.0, 0.5]])


def _entry(**extra):
    return {"observation_planes": ["horizontal", "vertical"],
            "observation_angles_deg": np.array([-45.0, 0.0, 45.0], np.float32), **extra}


def test_channel_basis_records():
    lf = np.array([[1 + 1j, 2, 1 - 1j], [0.5, 1, 0.5]], np.complex64)
    hf = np.array([[0.25, 0.5 + 0.5j, 0.25], [0.25, 0.25 + 0.25j, 0.25]], np.complex64)
    r = _frequency_result_from_channel_basis_entry(1000.0, _entry(source_results=[
        {"observation_pressure_complex": lf, "impedance": 1 + 0.5j, "lapack_info": 0, "backend": "test"},
        {"observation_pressure_complex": hf, "impedance": 2 - 0.25j, "lapack_info": 0, "backend": "test"}]),
        channel_names=np.asarray(["LF", "HF"]), channel_configs={})
    assert r.channel_names.tolist() == ["LF", "HF"]
    assert r.horizontal_pressure.shape == (2, 3) and r.vertical_pressure.shape == (2, 3)
    np.testing.assert_allclose(r.horizontal_pressure[0], np.conj(lf[0]))
    np.testing.assert_allclose(r.impedance, [[1.0, 0.5], [2.0, -0.25]])
    assert r.horizontal_spl_db.shape == (3,) and r.horizontal_spl_norm_db[1] == pytest.approx(0.0)
    # the synthesis with unit channel weights is the SPL of the summed (conjugated) basis
    np.testing.assert_allclose(r.horizontal_spl_db, 20 * np.log10(np.abs(lf[0] + hf[0]) / 20e-6), rtol=1e-5)
    sphere = np.array([1, 2, 3, 4], np.complex64)
    one = _frequency_result_from_channel_basis_entry(
        1000.0, _entry(observation_pressure_complex=lf, observation_sphere_pressure_complex=sphere, impedance=1.0),
        channel_names=np.asarray(["main"]), channel_configs={})
    assert one.sphere_pressure.shape == (1, 4)
    np.testing.assert_allclose(one.sphere_pressure[0], np.conj(sphere))
    none = _frequency_result_from_channel_basis_entry(1000.0, _entry(observation_pressure_complex=lf, impedance=1.0),
                                                      channel_names=np.asarray(["main"]), channel_configs={})
    assert none.sphere_pressure is None
    with pytest.raises(BoundaryLabSolverError, match="channel count"):
        _frequency_result_from_channel_basis_entry(1000.0, _entry(observation_pressure_complex=lf),
                                                   channel_names=np.asarray(["a", "b"]), channel_configs={})


def test_stream_resets_its_stop_flag_and_requires_frequencies():
    session = create_backend().create_session({"config": {"mesh_file": "m.msh"}})
    session._stop = True
    with pytest.raises(BoundaryLabSolverError, match="frequencies_hz"):
        next(session.solve_stream())
    assert session._stop is False
    with pytest.raises(BoundaryLabSolverError, match="SimulationConfig"):
        next(create_backend().create_session(None).solve_stream())


def test_stream_solves_one_unit_source_per_channel(monkeypatch):
    import hornlab_metal_bem_b200 as hb

    captured = {}
    lf = np.array([[1, 2, 1], [0.5, 1, 0.5]], np.complex64)
    hf = np.array([[0.25, 0.5, 0.25], [0.25, 0.25, 0.25]], np.complex64)

    def fake_solve_multi_source(mesh, sources, solve_config, frequencies_hz):
        captured.update(mesh=mesh, sources=sources, callback=solve_config.velocity_source_callback)
        entries = [{"observation_pressure_complex": lf if 7 in s else hf, "impedance": 1.0 if 7 in s else 2.0}
                   for s in sources]
        for i, f in enumerate(np.asarray(frequencies_hz)):
            if solve_config.on_frequency_result(i, float(f), _entry(source_results=entries)) is False:
                break
        return []

    monkeypatch.setattr(hb, "solve_multi_source", fake_solve_multi_source)
    config = SimpleNamespace(
        mesh_file="waveguide.msh", min_angle=-45.0, max_angle=45.0, step_size=45.0,
        radiators=(SimpleNamespace(name="woofer", tag=7, channel="LF", velocity_offset_db=6.0),
                   SimpleNamespace(name="tweeter", tag=8, channel="HF", velocity_offset_db=-6.0)),
        channels=(SimpleNamespace(name="LF"), SimpleNamespace(name="HF")))
    session = create_backend().create_session(SimpleNamespace(config=config, frequencies_hz=np.array([1000.0])))
    (result,) = list(session.solve_stream())
    assert captured["mesh"] == "waveguide.msh" and captured["callback"] is None
    assert captured["sources"][0][8] == pytest.approx(10.0 ** (-6.0 / 20.0))     # channels sorted: HF, LF
    assert captured["sources"][1][7] == pytest.approx(10.0 ** (6.0 / 20.0))
    assert result.channel_names.tolist() == ["HF", "LF"] and result.horizontal_pressure.shape == (2, 3)
    # a stop request makes the sweep's callback answer False, which ends the sweep after that frequency
    session = create_backend().create_session(SimpleNamespace(config=config, frequencies_hz=np.array([1e3, 2e3, 4e3])))
    got = list(session.solve_stream(stop_requested=lambda: True))
    assert [r.freq_hz for r in got] == [1000.0] and session._stop is True


def test_session_solve_routes_to_the_public_api(monkeypatch):
    import hornlab_metal_bem_b200 as hb

    calls = []
    monkeypatch.setattr(hb, "solve_frequencies", lambda mesh, f, cfg: calls.append(("freqs", mesh, list(f), cfg)) or "F")
    monkeypatch.setattr(hb, "solve", lambda mesh, cfg: calls.append(("grid", mesh, None, cfg)) or "G")
    s = create_backend(freq_count=5).create_session({"config": {"source_tag": 3}, "frequencies_hz": [500.0, 900.0]})
    assert s.solve("m.msh") == "F"
    kind, mesh, freqs, cfg = calls[-1]
    assert (kind, mesh, freqs) == ("freqs", "m.msh", [500.0, 900.0])
    assert cfg.velocity_sources == {3: 1.0} and cfg.freq_count == 5
    # an explicit config without frequencies solves on its own frequency grid
    assert s.solve("m.msh", {"frequency_count": 4}) == "G"
    assert calls[-1][0] == "grid" and calls[-1][3].freq_count == 5     # session overrides win
