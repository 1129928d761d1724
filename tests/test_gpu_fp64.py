"""The FP64 GPU path through the C ABI.

* ``hbem_assemble_f64`` / ``hbem_field_f64`` against the FP64 CPU oracle (the
  reference's corrected path restated in C, double precision): the same
  discretisation in the same precision, so they agree to rounding (1e-11).
* ``hbem_lu_factor_f64`` / ``hbem_lu_solve_f64`` against LAPACK zgesv: the
  same pivots (first maximum of |re| + |im|), solutions to 1e-12 on
  well-conditioned systems, a true FP64 solve where an FP32 factorisation and
  its refinement cannot reach (cond 1e9), info on a zero pivot.
* ``dense_solve_dtype="float64"`` end to end against the oracle.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import golden_buffers

from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a CUDA device", allow_module_level=True)

import hornlab_metal_bem_b200 as hb  # noqa: E402
from hornlab_metal_bem_b200 import generators as G  # noqa: E402
from hornlab_metal_bem_b200.native import (  # noqa: E402
    HBEM_PREC_PLAIN, HBEM_TRANS_N, NativeSession, _t_ptr, check, load_library, lu_solve_f64,
)

SYM = {"tiny": 0, "near": 0, "ico2": 0, "horn_quarter": 3, "yzxz_quarter": 3, "yz_half": 1, "xy_half": 4}


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


def _session(name):
    return NativeSession(golden_buffers(name), symmetry_plane={0: None, 1: "yz", 3: "yz+xz", 4: "xy"}[SYM[name]],
                         check_open_edges=False)


def _q(T, seed=0):
    rng = np.random.default_rng(seed)
    return (rng.normal(size=T) + 1j * rng.normal(size=T)).astype(np.complex64)


def _c(re, im):
    return re.cpu().numpy() + 1j * im.cpu().numpy()


@pytest.mark.parametrize("name", list(SYM))
@pytest.mark.parametrize("k", [1.8318326, 91.6, 366.366])
def test_f64_assembly_matches_fp64_oracle(name, k):
    b = golden_buffers(name)
    o = Oracle(b, SYM[name], "f64")
    q = _q(b.n_triangles)
    A_ref, b_ref = o.corrected(k, q)
    with _session(name) as s:
        Ar, Ai, br, bi = s.assemble_f64([k], q[None, :])
    assert rel(_c(Ar, Ai)[0], A_ref) < 1e-11
    assert rel(_c(br, bi)[0], b_ref) < 1e-11


def test_f64_complex_k_and_robin_match_fp64_oracle():
    b = golden_buffers("ico2")
    o = Oracle(b, 0, "f64")
    q = _q(b.n_triangles, 5)
    rng = np.random.default_rng(9)
    beta = np.where(rng.random(b.n_triangles) < 0.3, 0.4 + 0.2j, 0.0).astype(np.complex64)
    A_ref, b_ref = o.corrected(25.0, q, k_imag=0.125, beta=beta)
    with _session("ico2") as s:
        Ar, Ai, br, bi = s.assemble_f64([25.0], q[None, :], k_imag=[0.125], beta=beta)
    assert rel(_c(Ar, Ai)[0], A_ref) < 1e-11
    assert rel(_c(br, bi)[0], b_ref) < 1e-11


@pytest.mark.parametrize("name", ["ico2", "yzxz_quarter", "xy_half"])
def test_f64_field_matches_fp64_oracle(name):
    b = golden_buffers(name)
    o = Oracle(b, SYM[name], "f64")
    rng = np.random.default_rng(4)
    p = rng.normal(size=b.p1_dof_count) + 1j * rng.normal(size=b.p1_dof_count)
    q = rng.normal(size=b.n_triangles) + 1j * rng.normal(size=b.n_triangles)
    obs = (rng.normal(size=(3, 40)) * 1.5).astype(np.float32)
    obs[2] = np.abs(obs[2]) + 0.5
    ref = o.field(120.0, p, q, obs)
    with _session(name) as s:
        got = s.field_f64([120.0], p[None, :], q[None, :], obs).cpu().numpy()[0]
    assert rel(got, ref) < 1e-11


def _lu_case(n, batch, seed, nrhs=1):
    rng = np.random.default_rng(seed)
    A = rng.normal(size=(batch, n, n)) + 1j * rng.normal(size=(batch, n, n))
    A += np.eye(n)[None] * (0.5 * np.sqrt(n))
    b = rng.normal(size=(batch, n, nrhs)) + 1j * rng.normal(size=(batch, n, nrhs))
    return A, b


def _dev(z):
    return (torch.from_numpy(np.ascontiguousarray(z.real)).cuda(), torch.from_numpy(np.ascontiguousarray(z.imag)).cuda())


@pytest.mark.parametrize("n", [1, 2, 7, 31, 32, 33, 100, 257, 1043])
def test_f64_lu_matches_zgesv(n):
    from scipy.linalg import lapack

    A, b = _lu_case(n, 3, n)
    xr, xi = lu_solve_f64(*_dev(A), *_dev(b[..., 0]))
    x = _c(xr, xi)
    for m in range(3):
        ref = np.linalg.solve(A[m], b[m, :, 0])
        assert rel(x[m], ref) < 1e-11
    # pivots equal LAPACK's (first maximum of |re| + |im|)
    lib = load_library()
    Ar, Ai = _dev(A)
    piv = torch.empty((3, n), dtype=torch.int32, device="cuda")
    info = torch.empty(3, dtype=torch.int32, device="cuda")
    check(lib.hbem_lu_factor_f64(n, 3, _t_ptr(Ar), _t_ptr(Ai), n, n * n, _t_ptr(piv), n, _t_ptr(info), None),
          "hbem_lu_factor_f64", lib)
    for m in range(3):
        lu, ipiv, inf = lapack.zgetrf(A[m])
        assert inf == 0 and int(info[m]) == 0
        np.testing.assert_array_equal(piv[m].cpu().numpy(), ipiv)
        assert rel(_c(Ar, Ai)[m], lu) < 1e-11


def test_f64_lu_multiple_rhs_and_strides():
    A, b = _lu_case(150, 2, 11, nrhs=3)
    xr, xi = lu_solve_f64(*_dev(A), *_dev(b), nrhs=3)
    x = _c(xr, xi)
    for m in range(2):
        np.testing.assert_allclose(x[m], np.linalg.solve(A[m], b[m]), rtol=0, atol=1e-12 * np.abs(x[m]).max())


def test_f64_lu_zero_pivot_sets_info():
    lib = load_library()
    A, _ = _lu_case(40, 1, 3)
    A[0, :, 17] = 0.0   # column 17 is zero: the first zero pivot is at step 17
    Ar, Ai = _dev(A)
    piv = torch.empty((1, 40), dtype=torch.int32, device="cuda")
    info = torch.empty(1, dtype=torch.int32, device="cuda")
    check(lib.hbem_lu_factor_f64(40, 1, _t_ptr(Ar), _t_ptr(Ai), 40, 1600, _t_ptr(piv), 40, _t_ptr(info), None),
          "hbem_lu_factor_f64", lib)
    assert int(info[0]) == 18
    with pytest.raises(RuntimeError, match="zero pivot"):
        lu_solve_f64(*_dev(A), *_dev(np.ones((1, 40), complex)))


def test_f64_lu_solves_where_fp32_refinement_cannot():
    """cond(A) = 1e9 (singular values 1 .. 1e-9): beyond 1 / eps of FP32, so the FP32 factorisation and its
    FP64-residual refinement cannot recover the solution, while the complex128 LU does (the reason the reference
    offers zgesv)."""
    rng = np.random.default_rng(21)
    n = 200
    U, _ = np.linalg.qr(rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n)))
    V, _ = np.linalg.qr(rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n)))
    A = (U * np.logspace(0, -9, n)) @ V.conj().T
    x_true = rng.normal(size=n) + 1j * rng.normal(size=n)
    b = A @ x_true
    ref = np.linalg.solve(A, b)
    xr, xi = lu_solve_f64(*_dev(A[None]), *_dev(b[None]))
    e64 = rel(_c(xr, xi)[0], ref)
    assert e64 < 1e-5
    # FP32 LU + refinement on the same (rounded) system
    lib = load_library()
    A32 = A.astype(np.complex64)[None]
    Ar = torch.from_numpy(np.ascontiguousarray(A32.real)).cuda()
    Ai = torch.from_numpy(np.ascontiguousarray(A32.imag)).cuda()
    A0r, A0i = Ar.clone(), Ai.clone()
    br = torch.from_numpy(np.ascontiguousarray(b.real.astype(np.float32))[None]).cuda()
    bi = torch.from_numpy(np.ascontiguousarray(b.imag.astype(np.float32))[None]).cuda()
    x32r, x32i = br.clone(), bi.clone()
    piv = torch.empty((1, n), dtype=torch.int32, device="cuda")
    info = torch.empty(1, dtype=torch.int32, device="cuda")
    check(lib.hbem_lu_factor(n, 1, _t_ptr(Ar), _t_ptr(Ai), n, n * n, _t_ptr(piv), n, _t_ptr(info), HBEM_PREC_PLAIN,
                             None), "hbem_lu_factor", lib)
    check(lib.hbem_lu_solve(n, 1, 1, _t_ptr(Ar), _t_ptr(Ai), n, n * n, _t_ptr(piv), n, _t_ptr(x32r), _t_ptr(x32i), 1,
                            n, HBEM_TRANS_N, None), "hbem_lu_solve", lib)
    check(lib.hbem_refine(n, 1, _t_ptr(A0r), _t_ptr(A0i), n, n * n, _t_ptr(Ar), _t_ptr(Ai), n * n, _t_ptr(piv), n,
                          _t_ptr(br), _t_ptr(bi), n, _t_ptr(x32r), _t_ptr(x32i), n, 1e-12, 10, None, None, None),
          "hbem_refine", lib)
    e32 = rel(_c(x32r, x32i)[0], ref)
    assert e32 > 100 * e64


def test_dense_solve_dtype_float64_end_to_end():
    mesh = G.icosphere(3, 0.1)
    base = dict(freq_min_hz=1000.0, freq_max_hz=4000.0, freq_count=3, velocity_mode="velocity",
                return_surface_pressure=True)
    f64 = hb.solve(mesh, hb.native_config(dense_solve_dtype="float64", **base))
    plain = hb.solve(mesh, hb.native_config(**base))
    for f in range(3):
        a, b = f64.surface_pressure_complex[f], plain.surface_pressure_complex[f]
        assert rel(a, b) < 1e-5
        d = f64.native_diagnostics[f]
        assert d["dense_solve_impl"] == "hbem_blocked_lu_fp64"
        assert d["dense_solve_dtype"] == "float64"
        assert 0.0 < d["dense_solve_rcond"] < 1.0
        assert d["dense_solve_rcond"] == pytest.approx(plain.native_diagnostics[f]["dense_solve_rcond"], rel=0.05)
    assert np.max(np.abs(f64.directivity_db - plain.directivity_db)) < 1e-3


@pytest.mark.parametrize("name,sym,plane", [("ib_box", 0, None), ("ib_quarter_box", 3, "yz+xz")])
def test_f64_coupled_baffle_matches_fp64_oracle(name, sym, plane):
    """The coupled infinite baffle on the FP64 path (FP64 projections with their Duffy deltas, augmented
    complex128 solve, FP64 Rayleigh field) against the oracle's FP64 restatement of the reference's augmented
    solve (main.swift:7504-7595) and Rayleigh field (1397-1444)."""
    import ctypes

    buf = golden_buffers(name)
    obs = np.array([[0.0, 0.3, -0.2, 0.1, 0.0], [0.0, 0.1, 0.4, -0.3, 0.0], [2.0, 1.5, 0.8, 0.02, -0.5]],
                   np.float32)
    k = 2 * np.pi * 1500.0 / 343.0
    q = np.zeros((1, buf.n_triangles), np.complex64)
    q[0, buf.physical_tags_i32 == 2] = 1j * 1.2041 * 2 * np.pi * 1500.0
    o = Oracle(buf, sym, "f64")
    ap = o.aperture_triangles(7)
    A, b = o.corrected(k, q[0])
    p_ref, qa_ref, S_ia, S_aa = o.coupled_ib_solve(A, b, ap, k, k)
    f_ref = o.rayleigh(ap, k, qa_ref, obs)
    with NativeSession(buf, symmetry_plane=plane, aperture_tag=7, velocity_source_tags=[2],
                       check_open_edges=False) as s:
        n, m = s.n_dof, s.m_aperture
        sr = torch.empty((1, n, m), dtype=torch.float64, device="cuda")
        si = torch.empty_like(sr)
        ar = torch.empty((1, m, m), dtype=torch.float64, device="cuda")
        ai = torch.empty_like(ar)
        kk = np.array([k]), np.array([k])
        lib = load_library()
        assert lib.hbem_aperture_assemble_f64(s.handle, 1, kk[0].ctypes.data_as(ctypes.c_void_p), None,
                                              kk[1].ctypes.data_as(ctypes.c_void_p), _t_ptr(sr), _t_ptr(si),
                                              _t_ptr(ar), _t_ptr(ai), None) == 0
        assert rel(_c(sr, si)[0], S_ia) < 1e-11
        assert rel(_c(ar, ai)[0], S_aa) < 1e-11
        p, qa, fld = s.coupled_reference_solve_f64([k], q, obs)
    assert rel(p[0], p_ref) < 1e-9
    assert rel(qa[0], qa_ref) < 1e-9
    assert rel(fld[0], f_ref) < 1e-9
