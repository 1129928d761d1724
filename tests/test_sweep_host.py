"""Host logic of the sweep: per-frequency Robin admittance resolution (sweep.py:164-239 semantics)."""
from __future__ import annotations

import numpy as np
import pytest

import hornlab_metal_bem_b200 as hb
from hornlab_metal_bem_b200.sweep import impedance_sources_for_frequencies

TAGS = np.array([1, 1, 2, 2, 2], np.int32)


def test_static_admittance_skips_missing_tags():
    cfg = hb.native_config(impedance_sources={1: 0.3 + 0.1j, 9: 1.0})
    per = impedance_sources_for_frequencies(TAGS, [100.0, 200.0], cfg)
    assert per == [{1: 0.3 + 0.1j}, {1: 0.3 + 0.1j}]


def test_callback_overrides_and_extends_static():
    cfg = hb.native_config(impedance_sources={1: 0.5}, impedance_source_callback=lambda f: {2: f * 1e-3, 7: 1.0})
    per = impedance_sources_for_frequencies(TAGS, [100.0, 300.0], cfg)
    assert per == [{1: 0.5, 2: 0.1}, {1: 0.5, 2: 0.3}]
    cfg2 = hb.native_config(impedance_sources={1: 0.5}, impedance_source_callback=lambda f: {1: 0.25})
    assert impedance_sources_for_frequencies(TAGS, [50.0], cfg2) == [{1: 0.25}]


@pytest.mark.parametrize("bad", [-0.1, complex(float("nan"), 0.0)])
def test_callback_rejects_non_passive_or_non_finite(bad):
    cfg = hb.native_config(impedance_source_callback=lambda f: {1: bad})
    with pytest.raises(ValueError):
        impedance_sources_for_frequencies(TAGS, [100.0], cfg)


def test_case_flags_follow_the_reference_helper():
    """Per-case capability keys appear only when they apply, as the reference helper writes them
    (main.swift:9749-9761)."""
    from hornlab_metal_bem_b200.native import _case_flags

    assert _case_flags(3.0, 0.0) == {}
    assert _case_flags(3.0, 0.06) == {"assembly_k_imag_f32": 0.06, "complex_k": True}
    assert _case_flags(3.0, 0.0, robin=True) == {"robin_boundary": True, "field_uses_total_neumann": True}
    assert _case_flags(3.0, 0.0, robin=True, coupled=True) == {"robin_boundary": True}
    assert _case_flags(3.0, 0.0, coupled=True, field_k=3.0) == {}
    assert _case_flags(3.0, 0.0, coupled=True, field_k=2.5) == {"field_k_real_f32": 2.5}


def test_dense_solve_and_mesh_resolution_policies():
    """The per-frequency policy keys of the reference's sweep (tests/test_sweep_results.py:157-215)."""
    from types import SimpleNamespace

    from hornlab_metal_bem_b200.sweep import apply_dense_solve_policy, apply_mesh_resolution_policy, mesh_max_edge

    low = {"dense_solve_rcond": 1e-8}
    apply_dense_solve_policy(low, threshold=1e-6)
    assert low["dense_solve_rcond_warning_threshold"] == 1e-6
    assert low["dense_solve_suspect"] is True and low["dense_solve_policy_available"] is True
    assert "nudge or densify" in low["dense_solve_recommendation"]
    fine = {"dense_solve_rcond": 1e-2}
    apply_dense_solve_policy(fine, threshold=1e-6)
    assert fine["dense_solve_policy_available"] is True and fine["dense_solve_suspect"] is False
    unchecked = {}
    apply_dense_solve_policy(unchecked, threshold=1e-6)
    assert unchecked["dense_solve_policy_available"] is False and unchecked["dense_solve_suspect"] is False

    d = {}
    apply_mesh_resolution_policy(d, 1000.0, 0.1, 6.0)
    np.testing.assert_allclose(d["mesh_elements_per_wavelength"], 3.43)
    np.testing.assert_allclose(d["mesh_max_valid_frequency_hz"], 571.6666666666666)
    assert d["mesh_resolution_suspect"] is True

    mesh = SimpleNamespace(grid=SimpleNamespace(
        vertices=np.array([[0.0, 1.0, 0.0], [0.0, 0.0, 1.0], [0.0, 0.0, 0.0]]),
        elements=np.array([[0], [1], [2]], dtype=np.int32)))
    np.testing.assert_allclose(mesh_max_edge(mesh), np.sqrt(2.0))


def _fake_multi_source_env(monkeypatch):
    """Replace the GPU session and the single-source sweep with host fakes; returns the call log."""
    from contextlib import nullcontext

    import hornlab_metal_bem_b200.sweep as sw
    from hornlab_metal_bem_b200.result import MeshInfo, SolveResult

    calls = []

    def fake_run_sweep(mesh, frequencies, frame, config, *, session=None, average_tags=None):
        f = np.asarray(frequencies, dtype=np.float64)
        src = dict(config.velocity_sources)
        calls.append((tuple(f), src, tuple(average_tags or ()), config.on_frequency_result is None))
        base = float(sum(abs(v) * t for t, v in src.items()))
        p = (base + f[:, None, None] / 1000.0) * np.ones((f.size, 2, 3))
        log = [{"frequency_hz": float(x), "impedance": complex(base, x), "lapack_info": 0,
                "observation_sphere_pressure_complex": None} for x in f]
        return SolveResult(frequencies_hz=f, pressure_complex=p.astype(np.complex128), directivity_db=np.zeros_like(p),
                           impedance=np.array([complex(base, x) for x in f]), observation_angles_deg=np.array([-45.0, 0.0, 45.0]),
                           observation_points=np.zeros((2, 3, 3)), observation_planes=["horizontal", "vertical"],
                           config=config, mesh_info=MeshInfo(3, 1, {}, (np.zeros(3), np.ones(3))),
                           timings={"solve_s": 0.1 * f.size}, solver_log=log,
                           surface_pressure_avg={t: np.full(f.size, complex(t)) for t in (average_tags or src)},
                           native_diagnostics=[{"f": float(x)} for x in f])

    monkeypatch.setattr(sw, "run_sweep", fake_run_sweep)
    monkeypatch.setattr(sw, "NativeSession", lambda *a, **k: nullcontext(object()))
    return sw, calls


class _FakeBatchSession:
    """Host stand-in of a GPU session for the shared-factorisation multi-source sweep: each source's field is
    the sum of its Neumann row (so sources are told apart) plus f / 1000; every call is logged."""

    def __init__(self, calls):
        self.calls = calls

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        return False

    def assemble_solve_evaluate_standard_neumann_batch(self, freqs, k_re, q, pts, *, extra_neumann_dp0=None,
                                                       extra_impedance_source_tags=None, source_tags=None,
                                                       impedance_source_tag=None, **kw):
        from hornlab_metal_bem_b200.native import CaseResult, ExtraSourceResult

        freqs = np.atleast_1d(freqs)
        extra = np.zeros((0,) + np.shape(q)) if extra_neumann_dp0 is None else np.asarray(extra_neumann_dp0)
        self.calls.append((tuple(freqs), extra.shape, tuple(source_tags), impedance_source_tag,
                           tuple(extra_impedance_source_tags or ())))
        n_obs = pts.shape[1]
        out = []
        for f, fr in enumerate(freqs):
            def fields(row):
                return (np.abs(row).sum() + fr / 1000.0) * np.ones(n_obs, np.complex64)
            avg = {int(t): complex(t, fr) for t in source_tags}
            out.append(CaseResult(
                frequency_hz=float(fr), field=fields(q[f]), impedance=complex(np.abs(q[f]).sum(), fr),
                surface_pressure_avg=avg, surface_pressure=None, assembly_s=0.05, dense_solve_s=0.03, field_s=0.02,
                lapack_info=0, diagnostics={"f": float(fr), "dense_solve_rcond": 0.5},
                extra_sources=tuple(ExtraSourceResult(source_index=s + 1, field=fields(extra[s, f]),
                                                      impedance=complex(np.abs(extra[s, f]).sum(), fr),
                                                      surface_pressure_avg=avg, surface_pressure=None,
                                                      refine_iterations=1, refine_residual_rel=1e-8)
                                    for s in range(extra.shape[0]))))
        return out


def _two_tag_mesh_and_frame():
    from hornlab_metal_bem_b200 import generators as G
    from hornlab_metal_bem_b200.mesh import mesh_from_arrays
    from hornlab_metal_bem_b200.observation import infer_frame

    m = G.icosphere(1, 0.1)
    v, f = m.grid.vertices.T.copy(), m.grid.elements.T.copy()
    tags = np.where(v[f].mean(axis=1)[:, 2] < -0.05, 3, 2).astype(np.int32)
    mesh = mesh_from_arrays(v, f, tags, physical_groups={2: "2", 3: "3"})
    return mesh, infer_frame(mesh.grid, mesh.physical_tags, source_tag=2)


def test_multi_source_stream_interleaves_sources_per_frequency(monkeypatch):
    """With a streaming callback the shared-factorisation sweep runs one frequency per native call with every
    source as a right-hand side, and the callback sees one entry per frequency carrying ``source_results``
    (the reference's multi-RHS stream, sweep.py:1165-1210); False stops the sweep and the results keep the
    completed frequencies."""
    import hornlab_metal_bem_b200.sweep as sw

    calls = []
    monkeypatch.setattr(sw, "NativeSession", lambda *a, **k: _FakeBatchSession(calls))
    mesh, frame = _two_tag_mesh_and_frame()
    seen, progress = [], []

    def on_result(i, f, entry):
        seen.append((i, f, entry))
        return i < 1                       # stop after the second frequency

    cfg = hb.native_config(velocity_sources={2: 1.0}, on_frequency_result=on_result,
                           progress_callback=lambda i, n, f: progress.append((i, n, f)))
    sources = [{2: 1.0}, {2: 0.5, 3: 1.0}]
    out = sw.run_sweep_multi_source(mesh, [500.0, 1000.0, 2000.0], frame, cfg, sources)
    T = mesh.grid.number_of_elements
    assert [c[0] for c in calls] == [(500.0,), (1000.0,)]
    assert all(c[1] == (1, 1, T) and c[2] == (2, 3) and c[3] == 2 and c[4] == (2,) for c in calls)
    assert [(i, f) for i, f, _ in seen] == [(0, 500.0), (1, 1000.0)]
    assert progress == [(0, 3, 500.0), (1, 3, 1000.0)]
    e = seen[1][2]
    assert len(e["source_results"]) == 2 and e["impedance"] == e["source_results"][0]["impedance"]
    a0 = e["source_results"][0]["observation_pressure_complex"]
    a1 = e["source_results"][1]["observation_pressure_complex"]
    assert a0.shape == a1.shape and not np.allclose(a0, a1)
    assert e["observation_planes"] == cfg.observation.planes
    assert [r.frequencies_hz.tolist() for r in out] == [[500.0, 1000.0]] * 2
    assert set(out[1].surface_pressure_avg) == {2, 3}
    assert out[0].config.velocity_sources == {2: 1.0} and out[1].config.velocity_sources == {2: 0.5, 3: 1.0}
    assert out[1].native_diagnostics[0]["refine_iterations"] == 1 and out[1].native_diagnostics[0]["source_index"] == 1


def test_multi_source_without_stream_is_one_batch_for_all_sources(monkeypatch):
    """Without streaming every frequency and every source go into one native call (one assembly pass and one
    factorisation per frequency); each source gets its own result."""
    import hornlab_metal_bem_b200.sweep as sw

    calls = []
    monkeypatch.setattr(sw, "NativeSession", lambda *a, **k: _FakeBatchSession(calls))
    mesh, frame = _two_tag_mesh_and_frame()
    out = sw.run_sweep_multi_source(mesh, [500.0, 1000.0], frame, hb.native_config(), [{2: 1.0}, {3: 1.0}])
    T = mesh.grid.number_of_elements
    assert [(c[0], c[1], c[2]) for c in calls] == [((500.0, 1000.0), (1, 2, T), (2, 3))]
    assert len(out) == 2 and [r.config.velocity_sources for r in out] == [{2: 1.0}, {3: 1.0}]
    assert not np.allclose(out[0].pressure_complex, out[1].pressure_complex)


def test_multi_source_with_robin_walls_is_one_sweep_per_source(monkeypatch):
    sw, calls = _fake_multi_source_env(monkeypatch)
    mesh, frame = _two_tag_mesh_and_frame()
    cfg = hb.native_config(impedance_sources={3: 0.3 + 0.1j})
    out = sw.run_sweep_multi_source(mesh, [500.0, 1000.0], frame, cfg, [{2: 1.0}, {3: 1.0}])
    assert [(c[0], c[1], c[2]) for c in calls] == [((500.0, 1000.0), {2: 1.0}, (2, 3)),
                                                   ((500.0, 1000.0), {3: 1.0}, (2, 3))]
    assert len(out) == 2
    with pytest.raises(ValueError, match="at least one"):
        sw.run_sweep_multi_source(mesh, [500.0], frame, hb.native_config(), [])
    with pytest.raises(ValueError, match="velocity_source_callback"):
        sw.run_sweep_multi_source(mesh, [500.0], frame,
                                  hb.native_config(velocity_source_callback=lambda f: {2: 1.0}), [{2: 1.0}])


def test_near_quadrature_setting_parses_as_the_reference():
    """HORNLAB_METAL_BEM_NATIVE_NEAR_QUADRATURE values (main.swift:5024-5054): unset / '' / '0' = off, '1' /
    '2' = that level at threshold 1.5, '<level>:<threshold>'; anything else is rejected."""
    from hornlab_metal_bem_b200.native import parse_near_quadrature

    assert parse_near_quadrature(None) is None
    assert parse_near_quadrature("") is None and parse_near_quadrature("0") is None
    assert parse_near_quadrature("1") == (1, 1.5) and parse_near_quadrature("2") == (2, 1.5)
    assert parse_near_quadrature("2:1.25") == (2, 1.25)
    assert parse_near_quadrature((1, 2.0)) == (1, 2.0) and parse_near_quadrature((0, 1.0)) is None
    for bad in ("3", "1:0", "1:-2", "2:nan", "2:inf", "x", "1:2:3", "0:1.5"):
        with pytest.raises(ValueError, match="NEAR_QUADRATURE"):
            parse_near_quadrature(bad)
