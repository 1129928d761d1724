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
