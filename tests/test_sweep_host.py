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
