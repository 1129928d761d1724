"""CHIEF least squares on the GPU (``hbem_chief_lstsq``) against the oracle's restatement of the reference
(``main.swift:1897-2036`` rows, ``7186-7409`` zgels), and through ``solve()`` at the pulsating sphere's
fictitious frequency."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a CUDA device", allow_module_level=True)

import hornlab_metal_bem_b200 as hb  # noqa: E402
from hornlab_metal_bem_b200 import generators as G  # noqa: E402
from hornlab_metal_bem_b200.geometry import build_geometry_buffers  # noqa: E402
from hornlab_metal_bem_b200.mesh import make_pure_function_spaces  # noqa: E402
from hornlab_metal_bem_b200.native import NativeSession, _np_ptr, _stream_ptr, _t_ptr, check  # noqa: E402

from oracle.oracle import Oracle, chief_lstsq  # noqa: E402

PTS = np.array([[0.013, -0.021, 0.017], [-0.03, 0.02, -0.01], [0.025, 0.031, -0.028],
                [-0.012, -0.034, 0.03]], np.float64)          # (m, 3) inside the 0.1 m sphere
RHO, C0, A0 = 1.205, 343.0, 0.1


def _sphere(level=2):
    m = G.icosphere(level, A0)
    p1, dp0 = make_pure_function_spaces(m.grid)
    return m, build_geometry_buffers(m.grid, m.physical_tags, p1, dp0)


def _rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


@pytest.mark.parametrize("case", ["resonant", "plain", "robin", "two_sources"])
def test_chief_lstsq_matches_oracle_on_the_same_system(case):
    """The GPU's FP32-assembled A and b go through hbem_chief_lstsq and, copied to the host, through the
    oracle's FP64 CHIEF rows and LAPACK zgels: same solution (to the FP32 rounding of x), same scale s and
    the same chief_residual_rel."""
    _, buf = _sphere()
    T, n = buf.n_triangles, buf.p1_dof_count
    ka = 2.5 if case == "plain" else 3.18
    k = np.float32(ka / A0)
    rng = np.random.default_rng(7)
    qs = [np.full(T, 1j * RHO * float(k) * C0, np.complex64)]
    if case == "two_sources":
        qs.append((rng.normal(size=T) + 1j * rng.normal(size=T)).astype(np.complex64))
    beta = None
    if case == "robin":
        beta = np.full(T, 0.3 - 0.2j, np.complex64)
    S = len(qs)
    with NativeSession(buf, check_open_edges=False) as s:
        lib = s.lib
        bs = []
        for q in qs:
            Ar, Ai, br, bi = s.assemble(np.array([k]), q[None], beta=beta)
            bs.append((br[0], bi[0]))
        b_re = torch.stack([b[0] for b in bs]).contiguous()
        b_im = torch.stack([b[1] for b in bs]).contiguous()
        q_re = torch.tensor(np.stack([q.real for q in qs]).astype(np.float32), device="cuda")
        q_im = torch.tensor(np.stack([q.imag for q in qs]).astype(np.float32), device="cuda")
        be_re = be_im = None
        if beta is not None:
            be_re = torch.tensor(beta.real.astype(np.float32), device="cuda")
            be_im = torch.tensor(beta.imag.astype(np.float32), device="cuda")
        x_re = torch.empty((S, n), dtype=torch.float32, device="cuda")
        x_im = torch.empty_like(x_re)
        resid = torch.zeros(S, dtype=torch.float64, device="cuda")
        scale = torch.zeros(1, dtype=torch.float64, device="cuda")
        pts = np.ascontiguousarray(PTS.T, dtype=np.float32)
        kk = np.array([k], np.float32)
        check(lib.hbem_chief_lstsq(s.handle, 1, S, _np_ptr(kk), None, _t_ptr(q_re), _t_ptr(q_im), T, T,
                                   _t_ptr(be_re), _t_ptr(be_im), _t_ptr(Ar), _t_ptr(Ai), n, n * n, _t_ptr(b_re),
                                   _t_ptr(b_im), n, n, _np_ptr(pts), pts.shape[1], 1.0, _t_ptr(x_re), _t_ptr(x_im),
                                   n, n, _t_ptr(resid), _t_ptr(scale), _stream_ptr()), "hbem_chief_lstsq", lib)
        torch.cuda.synchronize()
        A = Ar[0].double().cpu().numpy() + 1j * Ai[0].double().cpu().numpy()
        B = (b_re.double().cpu().numpy() + 1j * b_im.double().cpu().numpy()).T     # (n, S)
        x = (x_re.double().cpu().numpy() + 1j * x_im.double().cpu().numpy()).T
        res = resid.cpu().numpy()
        sc = float(scale.cpu().numpy()[0])
    o = Oracle(buf, 0, "f64")
    Cm, D = None, []
    for q in qs:
        Cm, d, _ = o.chief_rows(pts, float(k), q, 0.0, beta)
        D.append(d)
    p, s_ref, res_ref = chief_lstsq(A, B, Cm, np.stack(D, axis=1), 1.0)
    assert abs(sc - s_ref) <= 1e-9 * s_ref
    for j in range(S):
        assert _rel(x[:, j], p[:, j]) < 2e-6
        assert abs(res[j] - res_ref[j]) <= 1e-4 * res_ref[j] + 1e-12


def _sphere_config(freqs, chief):
    return hb.native_config(
        freq_min_hz=float(freqs[0]), freq_max_hz=float(freqs[-1]), freq_count=len(freqs), freq_spacing="linear",
        velocity_mode="velocity",
        air_density=RHO, observation=hb.ObservationConfig(planes=["horizontal"], angle_count=13, distance_m=2.0),
        chief_points=PTS if chief else None,
    )


def test_solve_with_chief_points_cures_the_fictitious_frequency():
    """solve() at the ico2 sphere's near-singular ka = 3.18 (and ka = 2.5): with chief_points the impedance
    is the analytic pulsating sphere's to the discretisation error, without them it is 18 % off."""
    mesh, _ = _sphere()
    freqs = np.array([2.5, 3.18]) / A0 * C0 / (2 * np.pi)
    out = {}
    for chief in (False, True):
        out[chief] = hb.solve(mesh, _sphere_config(freqs, chief))
    res = out[True]
    k = (2 * np.pi * res.frequencies_hz / C0).astype(np.float32).astype(np.float64)
    za = RHO * C0 * (1j * k * A0) / (1j * k * A0 - 1)
    err_chief = np.abs(res.impedance - za) / np.abs(za)
    err_plain = np.abs(out[False].impedance - za) / np.abs(za)
    assert np.all(err_chief < 6e-3), err_chief
    assert err_plain[1] > 0.1 and err_plain[0] < 6e-3, err_plain
    diag = res.native_diagnostics[1]
    assert diag["chief_points"] is True and diag["dense_solve_dtype"] == "float64"
    assert 0 < diag["chief_residual_rel"] < 2e-2
