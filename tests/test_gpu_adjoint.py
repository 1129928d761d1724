"""Adjoint shape gradient against FP64 central finite differences.

The forward is the corrected P1 Neumann solve + exterior field; the objective
is the off-axis SPL deviation from a -6 dB / 60 degree target.  The finite
differences run the CPU oracle with FP64 arithmetic and FP64 vertex
coordinates (step 1e-6 m), i.e. the same discretisation in double precision.
Tolerance: the GPU forward and adjoint run in FP32 (matrix entries ~1e-6
relative, solves ~1e-5), so gradients agree to 2e-2 relative per control
point and 1e-2 relative as a vector.
"""
from __future__ import annotations

import numpy as np
import pytest

from oracle.oracle import Oracle, dense_solve

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a CUDA device", allow_module_level=True)

from hornlab_metal_bem_b200 import generators as G  # noqa: E402
from hornlab_metal_bem_b200.adjoint import (  # noqa: E402
    ShapeProblem, boundary_field, directivity_objective, directivity_points, spline_horn,
)
from hornlab_metal_bem_b200.geometry import build_geometry_buffers  # noqa: E402
from hornlab_metal_bem_b200.mesh import make_pure_function_spaces  # noqa: E402

ANGLES = [10, 20, 30, 40, 50, 60]


def _case(edge=0.025, freqs=(2000.0, 5000.0)):
    spec = G.horn_spec_from_seed(0, edge=edge)
    mesh, sh = spline_horn(spec, 24)
    p1, dp0 = make_pure_function_spaces(mesh.grid)
    buf = build_geometry_buffers(mesh.grid, mesh.physical_tags, p1, dp0)
    freqs = np.asarray(freqs)
    k = (2 * np.pi * freqs / 343.0).astype(np.float32)
    q = np.zeros((len(freqs), buf.triangles_3xm_i32.shape[1]), np.complex64)
    q[:, buf.physical_tags_i32 == 2] = 1.2041
    obs = directivity_points(spec.length, ANGLES).astype(np.float32)
    return buf, sh, k, q, obs


def _objective_f64(buf, sh, k, q, obs, c):
    o = Oracle(buf, 0, "g64", vertices_3xv=sh.vertices(c).T)
    field = []
    for f in range(len(k)):
        A, b = o.corrected(float(k[f]), q[f])
        p = dense_solve(A, b, "f64")
        field.append(o.field(float(k[f]), p, q[f], obs))
    return directivity_objective(np.asarray(field), ANGLES)


def test_adjoint_gradient_matches_fp64_finite_differences():
    buf, sh, k, q, obs = _case()
    c0 = np.random.default_rng(0).normal(0.0, 0.002, 24)
    prob = ShapeProblem(buf, k, q, obs)
    try:
        c = torch.tensor(c0, dtype=torch.float64, requires_grad=True)
        J = directivity_objective(boundary_field(sh.vertices(c), prob), ANGLES)
        J.backward()
        grad = c.grad.numpy()
    finally:
        prob.close()
    J64 = _objective_f64(buf, sh, k, q, obs, c0)
    assert abs(float(J.detach()) - J64) <= 1e-3 * abs(J64)
    h = 1e-6
    picks = [int(i) for i in np.argsort(-np.abs(grad))[:6]]
    fd = []
    for i in picks:
        e = np.zeros(24)
        e[i] = h
        fd.append((_objective_f64(buf, sh, k, q, obs, c0 + e) - _objective_f64(buf, sh, k, q, obs, c0 - e)) / (2 * h))
    fd = np.asarray(fd)
    got = grad[picks]
    assert np.linalg.norm(got - fd) <= 1e-2 * np.linalg.norm(fd), (got, fd)
    for g, r in zip(got, fd):
        assert abs(g - r) <= 2e-2 * abs(r) + 1e-3 * np.abs(fd).max(), (got, fd)


def test_adjoint_vertex_directional_derivative():
    """Every vertex moves (random direction): checks the field, assembly, Duffy
    and mass terms of the backward together, beyond the spline's wall motion."""
    buf, sh, k, q, obs = _case(freqs=(3000.0,))
    V = buf.vertices_3xn_f32.shape[1]
    base = np.asarray(buf.vertices_3xn_f32, dtype=np.float64).T
    rng = np.random.default_rng(1)
    direction = rng.normal(size=(V, 3))
    prob = ShapeProblem(buf, k, q, obs)
    try:
        v = torch.tensor(base, dtype=torch.float64, requires_grad=True)
        J = directivity_objective(boundary_field(v, prob), ANGLES)
        J.backward()
        dd = float((v.grad.numpy() * direction).sum())
    finally:
        prob.close()

    class Shift:
        def vertices(self, t):
            return base + t * direction

    sh2 = Shift()
    h = 1e-7
    fd = (_objective_f64(buf, sh2, k, q, obs, h) - _objective_f64(buf, sh2, k, q, obs, -h)) / (2 * h)
    assert abs(dd - fd) <= 2e-2 * abs(fd), (dd, fd)
