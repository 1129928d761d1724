"""Coupled infinite baffle on the GPU against the oracle's restatement of the
reference's augmented solve and Rayleigh field (main.swift:7504-7595,
1397-1444), and the quarter-vs-full known answer of the reference tests
(tests/test_metal_native.py:3849-3938: the yz+xz quadrant reproduces the
mirrored full box)."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import golden_buffers

from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a CUDA device", allow_module_level=True)

from hornlab_metal_bem_b200.native import NativeSession  # noqa: E402

RHO = 1.2041
OBS = np.array([[0.0, 0.3, -0.2, 0.1, 0.0], [0.0, 0.1, 0.4, -0.3, 0.0], [2.0, 1.5, 0.8, 0.02, -0.5]], np.float32)


def _q(buf, freqs):
    q = np.zeros((len(freqs), buf.n_triangles), np.complex64)
    for f, fr in enumerate(freqs):
        q[f, buf.physical_tags_i32 == 2] = 1j * RHO * 2 * np.pi * fr * 1.0
    return q


def _rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


@pytest.mark.parametrize("method", ["schur", "augmented"])
@pytest.mark.parametrize("name,sym,plane", [("ib_box", 0, None), ("ib_quarter_box", 3, "yz+xz")])
def test_coupled_ib_matches_oracle(name, sym, plane, method):
    buf = golden_buffers(name)
    freqs = np.array([300.0, 1500.0, 4000.0])
    k = (2 * np.pi * freqs / 343.0).astype(np.float32)
    q = _q(buf, freqs)
    with NativeSession(buf, symmetry_plane=plane, aperture_tag=7, velocity_source_tags=[2], check_open_edges=False) as s:
        # a two-frequency chunk limit exercises the chunked path (3 frequencies -> 2 + 1)
        n, m = s.n_dof, s.m_aperture
        per = 8 * ((n + m) ** 2 + n * m + m * m + 4 * (n + m)) if method == "augmented" else \
            8 * (n * n + 2 * n * m + 2 * m * m + 4 * n)
        res = s.coupled_ib_batch(freqs, k, q, OBS, source_tags=[2], impedance_source_tag=2, write_surface_pressure=True,
                                 coupled_method=method, max_chunk_bytes=2 * per)
    assert all(r.diagnostics["ib_coupled_solve"] == method for r in res)
    o = Oracle(buf, sym, "f64")
    ap = o.aperture_triangles(7)
    for f in range(len(freqs)):
        A, b = o.corrected(float(k[f]), q[f])
        p, qa, _, _ = o.coupled_ib_solve(A, b, ap, float(k[f]), float(k[f]))
        fld = o.rayleigh(ap, float(k[f]), qa, OBS)
        assert res[f].lapack_info == 0
        assert _rel(res[f].surface_pressure, p) < 1e-4
        assert _rel(res[f].diagnostics["aperture_neumann"], qa) < 1e-4
        assert _rel(res[f].field, fld) < 1e-4
        assert res[f].field[-1] == 0  # below the baffle


def test_quarter_box_equals_mirrored_full_box():
    quarter, full = golden_buffers("ib_quarter_box"), golden_buffers("ib_quarter_box_full")
    freqs = np.array([800.0, 2500.0])
    k = (2 * np.pi * freqs / 343.0).astype(np.float32)
    obs = np.array([[0.0, 0.05, 0.3], [0.0, 0.02, 0.1], [1.0, 0.5, 0.7]], np.float32)
    with NativeSession(quarter, symmetry_plane="yz+xz", aperture_tag=7, velocity_source_tags=[2],
                       check_open_edges=True) as sq:
        rq = sq.coupled_ib_batch(freqs, k, _q(quarter, freqs), obs, source_tags=[2], impedance_source_tag=2)
    with NativeSession(full, aperture_tag=7, velocity_source_tags=[2]) as sf:
        rf = sf.coupled_ib_batch(freqs, k, _q(full, freqs), obs, source_tags=[2], impedance_source_tag=2)
    for f in range(2):
        assert _rel(rq[f].field, rf[f].field) < 5e-4
        assert abs(rq[f].impedance - rf[f].impedance) / abs(rf[f].impedance) < 5e-4


def test_baffled_horn_augmented_matches_schur_and_mixed_refines():
    """Generated coupled-baffle horn (aperture of ~1000 faces, where the augmented
    system is the default): augmented == Schur, and BF16x3 + refinement == plain."""
    from hornlab_metal_bem_b200 import generators as G
    from hornlab_metal_bem_b200.native import AUGMENTED_MIN_APERTURE
    from hornlab_metal_bem_b200.geometry import build_geometry_buffers
    from hornlab_metal_bem_b200.mesh import make_pure_function_spaces

    spec = G.HornSpec(edge=0.012)
    mesh = G.baffled_horn(spec, aperture_tag=12)
    p1, dp0 = make_pure_function_spaces(mesh.grid)
    buf = build_geometry_buffers(mesh.grid, mesh.physical_tags, p1, dp0)
    freqs = np.array([1000.0, 6000.0])
    k = (2 * np.pi * freqs / 343.0).astype(np.float32)
    q = _q(buf, freqs)
    obs = np.array([[0.0, 0.5, 1.0], [0.0, 0.0, 0.5], [2.0, 1.5, 1.0]], np.float32)
    with NativeSession(buf, aperture_tag=12, velocity_source_tags=[2]) as s:
        assert s.m_aperture >= AUGMENTED_MIN_APERTURE
        kw = dict(source_tags=[2], impedance_source_tag=2, write_surface_pressure=True)
        ra = s.coupled_ib_batch(freqs, k, q, obs, **kw)
        rs = s.coupled_ib_batch(freqs, k, q, obs, coupled_method="schur", **kw)
        rm = s.coupled_ib_batch(freqs, k, q, obs, precision="mixed", refine_tolerance=1e-6, **kw)
    for f in range(2):
        assert ra[f].diagnostics["ib_coupled_solve"] == "augmented"
        assert _rel(ra[f].surface_pressure, rs[f].surface_pressure) < 1e-4
        assert _rel(ra[f].field, rs[f].field) < 1e-4
        assert rm[f].diagnostics["refine_residual_rel"] <= 1e-6
        assert _rel(rm[f].surface_pressure, ra[f].surface_pressure) < 1e-4
        assert _rel(rm[f].field, ra[f].field) < 1e-4
