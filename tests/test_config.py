"""Configuration surface of the drop-in API (host only): the defaults, the accepted values and the
rejections of ``SolveConfig`` / ``ObservationConfig`` that the reference's own unit tests pin
(tests/test_config.py:24-412, tests/test_hornlab_metal_bem_namespace.py:14-40), each rejection a
``ValueError`` naming the offending field."""
from __future__ import annotations

import numpy as np
import pytest

import hornlab_metal_bem_b200 as hb
from hornlab_metal_bem_b200.config import (
    AnnularProfile,
    BIEFormulation,
    CallableProfile,
    ObservationConfig,
    PerFaceProfile,
    SolveConfig,
    SourceMotion,
    TaperProfile,
)


def test_defaults():
    cfg = SolveConfig()
    assert cfg.formulation == BIEFormulation.STANDARD and cfg.complex_k_shift == 0.005
    assert cfg.impedance_sources == {} and cfg.impedance_source_callback is None
    assert cfg.native_symmetry_plane is None and cfg.native_check_open_edges is True
    assert cfg.metal_native_assembly_mode == "corrected" and cfg.return_surface_pressure is False
    for knob in ("metal_native_threads_per_group", "metal_native_matrix_threads_per_group",
                 "metal_native_rhs_threads_per_group", "metal_native_duffy_threads_per_group",
                 "metal_native_field_threads_per_group"):
        assert getattr(cfg, knob) is None
    assert cfg.dense_solve_rcond_warning_threshold == 1e-6 and cfg.mesh_elements_per_wavelength_min == 6.0
    assert cfg.mesh_validate is True and cfg.mesh_merge_tol == 1e-9 and cfg.mesh_repair_normals is False
    assert cfg.aperture_tag is None and cfg.frame_override is None
    assert cfg.air_density == 1.2041 and SolveConfig(air_density=1.18).air_density == 1.18
    assert cfg.progress_callback is None and cfg.on_frequency_result is None
    assert cfg.source_motion == SourceMotion.NORMAL and cfg.source_velocity_profiles is None
    assert ObservationConfig().custom_points is None
    nc = hb.native_config(freq_count=3)
    assert nc.metal_native_assembly_mode == "corrected" and nc.native_symmetry_plane is None and nc.freq_count == 3


def test_accepted_values():
    assert SolveConfig(source_motion=SourceMotion.AXIAL).source_motion == "axial"
    cfg = SolveConfig(source_velocity_profiles={
        2: TaperProfile(kind="linear", start=0.25), 3: AnnularProfile(0.2, 0.8),
        4: PerFaceProfile(np.array([1.0 + 0.0j])), 5: CallableProfile(lambda c, n, a, o: [1.0])})
    assert [type(p) for p in cfg.source_velocity_profiles.values()] == [TaperProfile, AnnularProfile,
                                                                         PerFaceProfile, CallableProfile]
    cfg = SolveConfig(formulation=BIEFormulation.COMPLEX_K, complex_k_shift=0.01,
                      impedance_sources={8: 0.05 + 0.01j, 9: 0.02 + 0.0j})
    assert cfg.formulation == "complex_k" and cfg.complex_k_shift == 0.01
    assert cfg.impedance_sources == {8: 0.05 + 0.01j, 9: 0.02 + 0.0j}
    for plane in ("yz", "xz", "xy", "yz+xz"):
        assert SolveConfig(native_symmetry_plane=plane).native_symmetry_plane == plane
    assert SolveConfig(native_check_open_edges=False).native_check_open_edges is False
    assert SolveConfig(aperture_tag=11).aperture_tag == 11
    for mode in ("corrected", "optimized", "reference", "parity"):
        assert SolveConfig(metal_native_assembly_mode=mode).metal_native_assembly_mode == mode
    assert SolveConfig(return_surface_pressure=True).return_surface_pressure is True
    assert SolveConfig(metal_native_threads_per_group=64).metal_native_threads_per_group == 64
    cfg = SolveConfig(metal_native_matrix_threads_per_group=32, metal_native_rhs_threads_per_group=64,
                      metal_native_duffy_threads_per_group=128, metal_native_field_threads_per_group=256)
    assert (cfg.metal_native_matrix_threads_per_group, cfg.metal_native_rhs_threads_per_group,
            cfg.metal_native_duffy_threads_per_group, cfg.metal_native_field_threads_per_group) == (32, 64, 128, 256)


REJECTED = [
    ({"freq_spacing": "octave"}, "freq_spacing"),
    ({"velocity_mode": "force"}, "velocity_mode"),
    ({"source_motion": "radial"}, "source_motion"),
    ({"source_velocity_profiles": {-1: TaperProfile()}}, "source_velocity_profiles tags"),
    ({"source_velocity_profiles": {2: "raised_cosine"}}, "SourceProfile"),
    ({"source_velocity_profiles": {2: TaperProfile(kind="hann")}}, "TaperProfile.kind"),
    ({"source_velocity_profiles": {2: TaperProfile(start=-0.1)}}, "TaperProfile.start"),
    ({"source_velocity_profiles": {2: TaperProfile(start=1.0)}}, "TaperProfile.start"),
    ({"source_velocity_profiles": {2: AnnularProfile(-0.1, 0.5)}}, "AnnularProfile"),
    ({"source_velocity_profiles": {2: AnnularProfile(0.7, 0.5)}}, "AnnularProfile"),
    ({"source_velocity_profiles": {2: AnnularProfile(0.0, 1.1)}}, "AnnularProfile"),
    ({"source_velocity_profiles": {2: PerFaceProfile([[1.0, 1.0]])}}, "PerFaceProfile.weights"),
    ({"source_velocity_profiles": {2: PerFaceProfile([complex(float("nan"), 0.0)])}}, "finite"),
    ({"source_velocity_profiles": {2: CallableProfile(None)}}, "CallableProfile.callback"),
    ({"formulation": "burton_miller"}, "formulation"),
    ({"complex_k_shift": -0.1}, "complex_k_shift"),
    ({"impedance_sources": {-1: 0.05 + 0.0j}}, "impedance_sources"),
    ({"impedance_sources": {8: complex(float("nan"), 0.0)}}, "impedance_sources"),
    ({"native_symmetry_plane": "zx"}, "native_symmetry_plane"),
    ({"freq_count": 0}, "freq_count"),
    ({"freq_min_hz": 0.0}, "freq_min_hz"),
    ({"freq_min_hz": -10.0}, "freq_min_hz"),
    ({"freq_min_hz": 1000.0, "freq_max_hz": 500.0}, "freq_max_hz"),
    ({"mesh_scale": 0.0}, "mesh_scale"),
    ({"air_density": 0.0}, "air_density"),
    ({"dense_solve_rcond_warning_threshold": -1.0}, "dense_solve_rcond_warning_threshold"),
    ({"mesh_elements_per_wavelength_min": 0.0}, "mesh_elements_per_wavelength_min"),
    ({"metal_native_assembly_mode": "unknown"}, "metal_native_assembly_mode"),
    ({"metal_native_threads_per_group": 0}, "metal_native_threads_per_group"),
] + [({"aperture_tag": bad}, "aperture_tag") for bad in (0, -1, True, 1.5, "11")] + [
    ({name: 0}, name) for name in ("metal_native_matrix_threads_per_group", "metal_native_rhs_threads_per_group",
                                   "metal_native_duffy_threads_per_group", "metal_native_field_threads_per_group")]


@pytest.mark.parametrize(("kwargs", "match"), REJECTED)
def test_solve_config_rejections(kwargs, match):
    with pytest.raises(ValueError, match=match):
        SolveConfig(**kwargs)


@pytest.mark.parametrize(("kwargs", "match"), [
    ({"planes": []}, "planes"), ({"distance_m": 0.0}, "distance_m"), ({"angle_count": 0}, "angle_count"),
    ({"origin": "Mouth"}, "origin"), ({"origin": "centre"}, "origin")])
def test_observation_config_rejections(kwargs, match):
    with pytest.raises(ValueError, match=match):
        ObservationConfig(**kwargs)


def test_public_namespace():
    for name in ("solve", "solve_frequencies", "native_config", "SolveConfig", "SolveResult", "SourceProfile",
                 "TaperProfile", "AnnularProfile", "PerFaceProfile", "CallableProfile", "load_mesh", "LoadedMesh"):
        assert name in hb.__all__, name
        assert getattr(hb, name) is not None
    for name in ("BIEFormulation", "LinearSolver", "DenseBieSystem"):
        assert name not in hb.__all__
