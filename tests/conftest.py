"""Shared fixtures: golden data loaders, GPU marker, repo on sys.path."""
from __future__ import annotations

import json
import sys
from pathlib import Path
from types import SimpleNamespace

import numpy as np
import pytest

REPO = Path(__file__).resolve().parent.parent
GOLDEN = REPO / "tests" / "golden"
if str(REPO) not in sys.path:
    sys.path.insert(0, str(REPO))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libhbem.so")
    config.addinivalue_line("markers", "slow: long CPU oracle runs")


def golden(name: str):
    return np.load(GOLDEN / name, allow_pickle=False)


def known_answers() -> dict:
    return json.loads((GOLDEN / "known_answers.json").read_text())


def golden_buffers(name: str):
    """Rebuild a GeometryBuffers from the golden geometry file."""
    from hornlab_metal_bem_b200.geometry import GeometryBuffers

    g = golden("geometry.npz")
    return GeometryBuffers(
        vertices_3xn_f32=g[f"{name}__vertices"],
        triangles_3xm_i32=g[f"{name}__triangles"],
        physical_tags_i32=g[f"{name}__tags"],
        p1_local2global_i32=g[f"{name}__l2g"],
        triangle_areas_f32=g[f"{name}__areas"],
        triangle_normals_3xm_f32=g[f"{name}__normals"],
        p1_dof_count=int(g[f"{name}__p1_count"]),
        dp0_dof_count=int(g[f"{name}__triangles"].shape[1]),
    )


def grid_from_buffers(b):
    return SimpleNamespace(
        vertices=np.asarray(b.vertices_3xn_f32, dtype=np.float64),
        elements=np.asarray(b.triangles_3xm_i32),
        number_of_elements=b.n_triangles,
    )


@pytest.fixture
def rng():
    return np.random.default_rng(1234)


def oracle_sweep(mesh, res, config, sym=0, systems=None):
    """The reference's corrected path in FP64 (oracle assembly, LAPACK zgesv, oracle field) at the
    frequencies of a ``SolveResult``: returns (surface pressure (F, n), field (F, N_obs)).  When a
    list is passed as ``systems``, each frequency's (A, b, q) is appended to it."""
    from hornlab_metal_bem_b200.bie import build_source_face_scale
    from hornlab_metal_bem_b200.geometry import build_geometry_buffers
    from hornlab_metal_bem_b200.mesh import make_pure_function_spaces
    from hornlab_metal_bem_b200.observation import infer_frame
    from hornlab_metal_bem_b200.sweep import field_points_3xn, k_values, neumann_rows
    from oracle.oracle import Oracle, dense_solve

    p1, dp0 = make_pure_function_spaces(mesh.grid)
    buf = build_geometry_buffers(mesh.grid, mesh.physical_tags, p1, dp0)
    o = Oracle(buf, sym, "f64")
    frame = infer_frame(mesh.grid, mesh.physical_tags, source_tag=min(config.velocity_sources),
                        symmetry_plane=config.native_symmetry_plane)
    scale = build_source_face_scale(mesh.grid, mesh.physical_tags, config, frame.axis, frame.source_center)
    k_re, _ = k_values(res.frequencies_hz, config)
    q = neumann_rows(buf.n_triangles, mesh.physical_tags, res.frequencies_hz, config, scale)
    pts = field_points_3xn(res.observation_points)
    beta = None
    if config.impedance_sources:
        beta = np.zeros(buf.n_triangles, np.complex64)
        for tag, bv in config.impedance_sources.items():
            beta[np.asarray(mesh.physical_tags) == int(tag)] = complex(bv)
    l2g = np.asarray(buf.p1_local2global_i32)
    out_p, out_f = [], []
    for f in range(len(res.frequencies_hz)):
        A, b = o.corrected(float(k_re[f]), q[f], 0.0, beta)
        p = dense_solve(A, b, "f64")
        if systems is not None:
            systems.append((A, b, q[f]))
        out_p.append(p)
        q_f = q[f].astype(np.complex128)
        if beta is not None:
            # the field's Neumann data on Robin faces: q + i k beta p_avg (main.swift:1646-1674)
            q_f = q_f + 1j * float(k_re[f]) * beta * p[l2g].mean(axis=1)
        out_f.append(o.field(float(k_re[f]), p, q_f, pts))
    return np.array(out_p), np.array(out_f)
