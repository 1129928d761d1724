"""GPU parity: every CUDA stage through the C ABI against the CPU oracle.

Tolerances (the path's accuracy targets): assembled matrix and RHS within 1e-4
relative L2 of the reference method (here the FP64 oracle, which is pinned to
the reference's known answers in test_oracle_pins.py); LU solutions within
1e-5 of LAPACK; field within 1e-4 relative; directivity within 0.01 dB.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from conftest import golden_buffers

from oracle.oracle import Oracle, dense_solve

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover - CPU containers
    pytest.skip("needs a CUDA device", allow_module_level=True)

from hornlab_metal_bem_b200 import generators as G  # noqa: E402
from hornlab_metal_bem_b200.geometry import build_geometry_buffers  # noqa: E402
from hornlab_metal_bem_b200.mesh import make_pure_function_spaces  # noqa: E402
from hornlab_metal_bem_b200.native import (  # noqa: E402
    HBEM_ASM_CORRECTED, HBEM_ASM_REGULAR, HBEM_ASM_ZERO, HBEM_TRANS_N, NativeSession, _t_ptr, last_error,
    load_library,
)

HBEM_ERR_STATE = -4
HBEM_TUNE_LU_SOLVE, HBEM_TUNE_WAVE_SPIN = 2, 7

SYM = {"tiny": 0, "near": 0, "ico2": 0, "horn_quarter": 3, "yzxz_quarter": 3, "yzxz_full": 0, "yz_half": 1,
       "xy_half": 4, "ib_box": 0, "yz_full": 0}


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


def _session(name):
    return NativeSession(golden_buffers(name), symmetry_plane={0: None, 1: "yz", 3: "yz+xz", 4: "xy"}[SYM[name]],
                         check_open_edges=False)


def _q(T, seed=0):
    rng = np.random.default_rng(seed)
    return (rng.normal(size=T) + 1j * rng.normal(size=T)).astype(np.complex64)


def _host(t_re, t_im):
    return t_re.cpu().numpy().astype(np.float64) + 1j * t_im.cpu().numpy().astype(np.float64)


@pytest.mark.parametrize("name", ["tiny", "near", "ico2", "horn_quarter", "yzxz_quarter", "yz_half", "xy_half"])
@pytest.mark.parametrize("k", [1.8318326, 18.3, 91.6, 250.0, 366.366])
def test_corrected_assembly_matches_oracle(name, k):
    """k up to 366.366 rad/m: 20 kHz, the top of the benchmark sweep."""
    b = golden_buffers(name)
    o = Oracle(b, SYM[name], "f64")
    q = _q(b.n_triangles)
    A_ref, b_ref = o.corrected(k, q)
    with _session(name) as s:
        Ar, Ai, br, bi = s.assemble([k], q[None, :])
        A, rhs = _host(Ar, Ai)[0], _host(br, bi)[0]
    assert rel(A, A_ref) < 1e-4
    assert rel(rhs, b_ref) < 1e-4


@pytest.mark.parametrize("name", ["ico2", "horn_quarter"])
def test_regular_only_assembly_matches_oracle(name):
    b = golden_buffers(name)
    o = Oracle(b, SYM[name], "f64")
    q = _q(b.n_triangles, 3)
    A_ref, b_ref = o.regular(40.0, q)
    with _session(name) as s:
        Ar, Ai, br, bi = s.assemble([40.0], q[None, :], flags=HBEM_ASM_REGULAR | HBEM_ASM_ZERO)
    assert rel(_host(Ar, Ai)[0], A_ref) < 1e-4
    assert rel(_host(br, bi)[0], b_ref) < 1e-4


def test_complex_k_and_robin_assembly_match_oracle():
    b = golden_buffers("ico2")
    o = Oracle(b, 0, "f64")
    q = _q(b.n_triangles, 5)
    rng = np.random.default_rng(9)
    beta = np.where(rng.random(b.n_triangles) < 0.3, 0.4 + 0.2j, 0.0).astype(np.complex64)
    A_ref, b_ref = o.corrected(25.0, q, k_imag=0.125, beta=beta)
    with _session("ico2") as s:
        Ar, Ai, br, bi = s.assemble([25.0], q[None, :], k_imag=[0.125], beta=beta)
    assert rel(_host(Ar, Ai)[0], A_ref) < 1e-4
    assert rel(_host(br, bi)[0], b_ref) < 1e-4


def test_multi_frequency_batch_equals_single_frequency():
    b = golden_buffers("horn_quarter")
    ks = [3.0, 20.0, 75.0]
    q = np.stack([_q(b.n_triangles, i) for i in range(3)])
    with _session("horn_quarter") as s:
        Ar, Ai, br, bi = s.assemble(ks, q)
        for f, k in enumerate(ks):
            Ar1, Ai1, br1, bi1 = s.assemble([k], q[f][None, :])
            assert rel(_host(Ar, Ai)[f], _host(Ar1, Ai1)[0]) < 1e-6
            assert rel(_host(br, bi)[f], _host(br1, bi1)[0]) < 1e-6


@pytest.mark.parametrize("name", ["tiny", "ico2", "horn_quarter", "yzxz_quarter"])
def test_pair_plan_matches_oracle(name):
    b = golden_buffers(name)
    o = Oracle(b, SYM[name], "f64")
    pairs, counts = o.duffy_pairs()
    with _session(name) as s:
        plan = s.pair_plan()
        assert {k: plan[k] for k in counts} == counts
        assert s.query("unique_triplets") == o.unique_triplets(pairs)
        assert s.query("image_pairs") == int(np.sum((pairs[:, 2] != 0) | (pairs[:, 3] != 0)))


def test_quarter_equals_orbit_reduced_full_on_gpu():
    with _session("yzxz_full") as sf, _session("yzxz_quarter") as sq:
        Af = _host(*sf.assemble([1.8318326], np.ones((1, 4), np.complex64))[:2])[0]
        bf = _host(*sf.assemble([1.8318326], np.ones((1, 4), np.complex64))[2:])[0]
        Aq_r, Aq_i, bq_r, bq_i = sq.assemble([1.8318326], np.ones((1, 1), np.complex64))
    orbits = [np.array([0]), np.array([1, 3]), np.array([2, 4])]
    R = np.array([[Af[np.ix_(r, c)].sum() for c in orbits] for r in orbits])
    rb = np.array([bf[r].sum() for r in orbits])
    assert rel(_host(Aq_r, Aq_i)[0], R) < 1e-6
    assert rel(_host(bq_r, bq_i)[0], rb) < 1e-6


# ---------------------------------------------------------------------------- LU
def _lu_case(n, batch, seed):
    rng = np.random.default_rng(seed)
    A = rng.normal(size=(batch, n, n)) + 1j * rng.normal(size=(batch, n, n))
    A += np.eye(n)[None] * (2.0 * np.sqrt(n))
    b = rng.normal(size=(batch, n)) + 1j * rng.normal(size=(batch, n))
    return A.astype(np.complex64), b.astype(np.complex64)


def _dev(z):
    return (torch.from_numpy(np.ascontiguousarray(z.real, np.float32)).cuda(),
            torch.from_numpy(np.ascontiguousarray(z.imag, np.float32)).cuda())


def _factor(Ar, Ai, n, batch, precision=0):
    import ctypes

    lib = load_library()
    piv = torch.zeros((batch, n), dtype=torch.int32, device="cuda")
    info = torch.zeros(batch, dtype=torch.int32, device="cuda")
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = lib.hbem_lu_factor(n, batch, ctypes.c_void_p(Ar.data_ptr()), ctypes.c_void_p(Ai.data_ptr()), n, n * n,
                            ctypes.c_void_p(piv.data_ptr()), n, ctypes.c_void_p(info.data_ptr()), precision, st)
    assert rc == 0
    return piv, info


def _solve(Ar, Ai, piv, Br, Bi, n, nrhs, batch, trans=0):
    import ctypes

    lib = load_library()
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = lib.hbem_lu_solve(n, nrhs, batch, ctypes.c_void_p(Ar.data_ptr()), ctypes.c_void_p(Ai.data_ptr()), n, n * n,
                           ctypes.c_void_p(piv.data_ptr()), n, ctypes.c_void_p(Br.data_ptr()),
                           ctypes.c_void_p(Bi.data_ptr()), nrhs, n * nrhs, trans, st)
    assert rc == 0


@pytest.mark.parametrize("n", [1, 2, 5, 31, 33, 100, 257, 700, 1059])
def test_lu_solve_matches_lapack(n):
    batch = 3
    A, b = _lu_case(n, batch, n)
    Ar, Ai = _dev(A)
    piv, info = _factor(Ar, Ai, n, batch)
    assert int(info.abs().sum()) == 0
    Br, Bi = _dev(b[:, :, None])
    _solve(Ar, Ai, piv, Br, Bi, n, 1, batch)
    x = _host(Br, Bi)[:, :, 0]
    for m in range(batch):
        ref = np.linalg.solve(A[m].astype(np.complex128), b[m].astype(np.complex128))
        assert rel(x[m], ref) < 1e-5


@pytest.mark.parametrize("trans", [0, 2])
def test_wavefront_solve_many_matrices(trans):
    """More 32-row blocks than resident CTAs (40 matrices of n = 1043): the wavefront solve against LAPACK
    and against the one-CTA-per-right-hand-side scheme."""
    lib = load_library()
    n, batch = 1043, 40
    A, b = _lu_case(n, batch, 5)
    Ar, Ai = _dev(A)
    piv, info = _factor(Ar, Ai, n, batch)
    assert int(info.abs().sum()) == 0
    out = {}
    for mode in (3, 1):
        Br, Bi = _dev(b[:, :, None])
        assert lib.hbem_set_tuning(2, mode) == 0
        try:
            _solve(Ar, Ai, piv, Br, Bi, n, 1, batch, trans)
        finally:
            lib.hbem_set_tuning(2, 0)
        out[mode] = _host(Br, Bi)[:, :, 0]
    assert np.isfinite(out[3]).all()
    assert rel(out[3], out[1]) < 1e-5
    for m in (0, 17, 39):
        op = A[m] if trans == 0 else A[m].conj().T
        ref = np.linalg.solve(op.astype(np.complex128), b[m].astype(np.complex128))
        assert rel(out[3][m], ref) < 1e-5


@pytest.mark.parametrize("panel", [32, 64])
def test_lu_bitwise_stable_under_concurrent_work(panel):
    """The factorisation of matrices whose first panels span thread-block clusters (n = 1043: 2 CTAs for
    32-wide sub-panels, 4 for whole 64-column blocks) must not depend on what else runs on the GPU: a
    matrix-multiply load on another stream changes CTA timing, which once exposed a missing barrier between
    a panel's last scaling pass and its write-back."""
    lib = load_library()
    n, batch = 1043, 40
    A, _ = _lu_case(n, batch, 17)
    A0r, A0i = _dev(A)
    side = torch.cuda.Stream()
    X = torch.randn(4096, 4096, device="cuda")
    runs = []
    assert lib.hbem_set_tuning(1, panel) == 0
    try:
        for noisy in (False, True, True, True):
            Ar, Ai = A0r.clone(), A0i.clone()
            torch.cuda.synchronize()
            if noisy:
                with torch.cuda.stream(side):
                    for _ in range(60):
                        X @ X
            piv, info = _factor(Ar, Ai, n, batch)
            torch.cuda.synchronize()
            runs.append((Ar, Ai, piv, info))
    finally:
        lib.hbem_set_tuning(1, 0)
    assert int(runs[0][3].abs().sum()) == 0
    for r in runs[1:]:
        assert all(torch.equal(x, y) for x, y in zip(runs[0][:3], r[:3]))
    # and the factors are right: P A = L U for one matrix
    LU = _host(runs[0][0], runs[0][1])[5]
    pv = runs[0][2][5].cpu().numpy()
    PA = A[5].astype(np.complex128).copy()
    for k in range(n):
        if pv[k] != k:
            PA[[k, pv[k]]] = PA[[pv[k], k]]
    L = np.tril(LU, -1) + np.eye(n)
    assert rel(L @ np.triu(LU), PA) < 1e-5


@pytest.mark.parametrize("precision", [0, 1])
def test_lu_tall_panels_sixteen_cta_clusters(precision):
    """n = 12200: the first 16-column panels (over 12 047 rows) outgrow an 8-CTA cluster's shared memory and
    are factored in 16-CTA clusters.  The pivot is the first maximum of |re| + |im|, which bounds every
    multiplier's modulus by sqrt(2); and the factors solve the system (residual in FP64)."""
    import ctypes

    lib = load_library()
    n = 12200
    g = torch.Generator(device="cuda").manual_seed(5)
    A0r = torch.randn((1, n, n), device="cuda", generator=g)
    A0i = torch.randn((1, n, n), device="cuda", generator=g)
    Ar, Ai = A0r.clone(), A0i.clone()
    piv, info = _factor(Ar, Ai, n, 1, precision)
    torch.cuda.synchronize()
    assert int(info.abs().sum()) == 0
    low = torch.tril(torch.hypot(Ar[0], Ai[0]), -1)
    assert float(low.max()) <= 2 ** 0.5 * (1 + 1e-6)
    del low
    br = torch.randn((1, n), device="cuda", generator=g)
    bi = torch.randn((1, n), device="cuda", generator=g)
    xr, xi = br.clone(), bi.clone()
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    P = lambda t: ctypes.c_void_p(t.data_ptr())
    assert lib.hbem_lu_solve(n, 1, 1, P(Ar), P(Ai), n, n * n, P(piv), n, P(xr), P(xi), 1, n, 0, st) == 0
    torch.cuda.synchronize()
    A = torch.complex(A0r[0].double(), A0i[0].double())
    x = torch.complex(xr[0].double(), xi[0].double())
    b = torch.complex(br[0].double(), bi[0].double())
    r = float(torch.linalg.norm(A @ x - b) / (torch.linalg.norm(A) * torch.linalg.norm(x)))
    # normwise backward error: FP32 updates, or BF16x3 ones (16 significand bits per operand)
    assert r < (1e-5 if precision == 0 else 1e-4)


@pytest.mark.parametrize("n,batch", [(1043, 12), (2100, 3)])
def test_lu_lookahead_equals_one_stream(n, batch):
    """The look-ahead schedule (next block updated on the chain, the rest of the trailing update overlapping the
    next panels on a second stream) does the same arithmetic in the same order: bit-identical factors (with the
    CUDA-core update in both; the tensor-core bulk exists only beside a look-ahead chain)."""
    lib = load_library()
    A, _ = _lu_case(n, batch, 23)
    out = []
    for mode in (1, 0, 0):
        Ar, Ai = _dev(A)
        assert lib.hbem_set_tuning(5, mode) == 0
        assert lib.hbem_set_tuning(8, 1) == 0
        try:
            piv, info = _factor(Ar, Ai, n, batch)
        finally:
            lib.hbem_set_tuning(5, 0)
            lib.hbem_set_tuning(8, 0)
        torch.cuda.synchronize()
        out.append((Ar, Ai, piv))
    for r in out[1:]:
        assert all(torch.equal(x, y) for x, y in zip(out[0], r))


@pytest.mark.parametrize("n", [1800, 3300, 6500])
def test_lu_tall_panels_match_lapack(n):
    """Sizes whose sub-panels spread over 2-, 4- and 8-CTA clusters, two right-hand sides."""
    batch, nrhs = 1, 2
    A, _ = _lu_case(n, batch, n)
    rng = np.random.default_rng(n + 1)
    B = (rng.normal(size=(batch, n, nrhs)) + 1j * rng.normal(size=(batch, n, nrhs))).astype(np.complex64)
    Ar, Ai = _dev(A)
    piv, info = _factor(Ar, Ai, n, batch)
    assert int(info.abs().sum()) == 0
    Br, Bi = _dev(B)
    _solve(Ar, Ai, piv, Br, Bi, n, nrhs, batch)
    X = _host(Br, Bi)
    ref = np.linalg.solve(A[0].astype(np.complex128), B[0].astype(np.complex128))
    # FP32 factorisation error grows with n; LAPACK cgesv in FP32 shows the same
    assert rel(X[0], ref) < (1e-5 if n < 3000 else 3e-5)


@pytest.mark.parametrize("n,panel", [(1043, 0), (1300, 0), (700, 16), (1043, 32)])
def test_register_panel_matches_shared_memory_panel(n, panel):
    """Sub-panels with their rows in registers (HBEM_TUNE_LU_PANEL_KERNEL = 1: 64 columns x 384 rows,
    32 x 768, 16 x 1024) give the same pivots and the same factors, bit for bit, as the shared-memory panel
    kernel at the same sub-panel widths; HBEM_TUNE_LU_PANEL = 16 or 32 fixes the width in every block."""
    lib = load_library()
    batch = 5
    A, _ = _lu_case(n, batch, n + 11)
    out = {}
    assert lib.hbem_set_tuning(1, panel) == 0
    try:
        for kernel in (0, 1):
            Ar, Ai = _dev(A)
            assert lib.hbem_set_tuning(10, kernel) == 0
            piv, info = _factor(Ar, Ai, n, batch)
            torch.cuda.synchronize()
            out[kernel] = (Ar, Ai, piv, info)
    finally:
        lib.hbem_set_tuning(10, 0)
        lib.hbem_set_tuning(1, 0)
    assert int(out[0][3].abs().sum()) == 0 and int(out[1][3].abs().sum()) == 0
    assert torch.equal(out[0][2], out[1][2])
    assert torch.equal(out[0][0], out[1][0]) and torch.equal(out[0][1], out[1][1])


@pytest.mark.parametrize("n,batch", [(1043, 6), (1542, 3)])
def test_tf32x3_precision_refined_matches_lapack(n, batch):
    """HBEM_PREC_TF32X3 (the FP32 LU with its bulk update on the tensor cores) followed by FP64-residual
    refinement reaches the refinement tolerance and LAPACK's complex128 solution."""
    lib = load_library()
    A, b = _lu_case(n, batch, n + 3)
    A0r, A0i = _dev(A)
    Ar, Ai = A0r.clone(), A0i.clone()
    piv, info = _factor(Ar, Ai, n, batch, precision=3)
    assert int(info.abs().sum()) == 0
    br, bi = _dev(b)
    xr, xi = br.clone(), bi.clone()
    _solve(Ar, Ai, piv, xr.view(batch, n, 1), xi.view(batch, n, 1), n, 1, batch)
    iters = torch.zeros(batch, dtype=torch.int32, device="cuda")
    resid = torch.zeros(batch, dtype=torch.float64, device="cuda")
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    p = ctypes.c_void_p
    rc = lib.hbem_refine(n, batch, p(A0r.data_ptr()), p(A0i.data_ptr()), n, n * n, p(Ar.data_ptr()), p(Ai.data_ptr()),
                         n * n, p(piv.data_ptr()), n, p(br.data_ptr()), p(bi.data_ptr()), n, p(xr.data_ptr()),
                         p(xi.data_ptr()), n, ctypes.c_double(1e-7), 5, p(iters.data_ptr()), p(resid.data_ptr()), st)
    assert rc == 0
    assert float(resid.max()) <= 1e-7
    x = _host(xr, xi)
    for m in range(batch):
        ref = np.linalg.solve(A[m].astype(np.complex128), b[m].astype(np.complex128))
        assert rel(x[m], ref) < 1e-6


@pytest.mark.parametrize("n,batch,kpass", [(300, 3, 0), (1043, 6, 0), (3300, 1, 0), (1043, 6, 64), (3300, 1, 64)])
def test_plain_lu_tensor_core_update_matches_lapack(n, batch, kpass):
    """The plain LU with its look-ahead bulk update on the tensor cores (TF32x3 split products,
    HBEM_TUNE_LU_UPDATE = 2) against LAPACK and against the CUDA-core (exact FP32 product) update; the
    bulk in two K = 32 passes per 64-column block (built in below n = 12000) and in one K = 64 pass
    (HBEM_TUNE_LU_BLOCK = 64)."""
    lib = load_library()
    A, b = _lu_case(n, batch, n + 7)
    xs = {}
    for mode in (1, 2):
        Ar, Ai = _dev(A)
        assert lib.hbem_set_tuning(8, mode) == 0
        assert lib.hbem_set_tuning(9, kpass) == 0
        try:
            piv, info = _factor(Ar, Ai, n, batch)
        finally:
            lib.hbem_set_tuning(8, 0)
            lib.hbem_set_tuning(9, 0)
        assert int(info.abs().sum()) == 0
        Br, Bi = _dev(b[:, :, None])
        _solve(Ar, Ai, piv, Br, Bi, n, 1, batch)
        xs[mode] = _host(Br, Bi)[:, :, 0]
    for m in range(batch):
        ref = np.linalg.solve(A[m].astype(np.complex128), b[m].astype(np.complex128))
        assert rel(xs[2][m], ref) < (1e-5 if n < 3000 else 3e-5)
        assert rel(xs[2][m], xs[1][m]) < (1e-5 if n < 3000 else 3e-5)


@pytest.mark.parametrize("n", [130, 700])
@pytest.mark.parametrize("trans", [1, 2])
def test_transposed_solves(trans, n):
    batch, nrhs = 2, 3
    A, _ = _lu_case(n, batch, 11)
    rng = np.random.default_rng(2)
    B = (rng.normal(size=(batch, n, nrhs)) + 1j * rng.normal(size=(batch, n, nrhs))).astype(np.complex64)
    Ar, Ai = _dev(A)
    piv, info = _factor(Ar, Ai, n, batch)
    Br, Bi = _dev(B)
    _solve(Ar, Ai, piv, Br, Bi, n, nrhs, batch, trans)
    X = _host(Br, Bi)
    for m in range(batch):
        op = A[m].T if trans == 1 else A[m].conj().T
        ref = np.linalg.solve(op.astype(np.complex128), B[m].astype(np.complex128))
        assert rel(X[m], ref) < 1e-5


@pytest.mark.parametrize("mode", [1, 2, 3])
@pytest.mark.parametrize("trans", [0, 1, 2])
@pytest.mark.parametrize("n", [33, 130, 700])
def test_solve_schemes_match_lapack(n, trans, mode):
    """Every solve scheme (1: one CTA per right-hand side, 2: blocked multi-CTA steps, 3: wavefront) for A, A^T, A^H."""
    lib = load_library()
    batch, nrhs = 2, 3
    A, _ = _lu_case(n, batch, 900 + n)
    rng = np.random.default_rng(n + trans)
    B = (rng.normal(size=(batch, n, nrhs)) + 1j * rng.normal(size=(batch, n, nrhs))).astype(np.complex64)
    Ar, Ai = _dev(A)
    piv, info = _factor(Ar, Ai, n, batch)
    Br, Bi = _dev(B)
    assert lib.hbem_set_tuning(2, mode) == 0
    try:
        _solve(Ar, Ai, piv, Br, Bi, n, nrhs, batch, trans)
    finally:
        lib.hbem_set_tuning(2, 0)
    X = _host(Br, Bi)
    for m in range(batch):
        op = A[m] if trans == 0 else (A[m].T if trans == 1 else A[m].conj().T)
        ref = np.linalg.solve(op.astype(np.complex128), B[m].astype(np.complex128))
        assert rel(X[m], ref) < 1e-5


def _rcond_gpu(A):
    """GPU ||A||_1 and cgecon-style estimate for a (batch, n, n) complex64 stack."""
    import ctypes

    lib = load_library()
    batch, n = A.shape[0], A.shape[1]
    Ar, Ai = _dev(A)
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    anorm = torch.empty(batch, dtype=torch.float32, device="cuda")
    P = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    assert lib.hbem_matrix_norm1(n, batch, P(Ar), P(Ai), n, n * n, P(anorm), st) == 0
    piv, info = _factor(Ar, Ai, n, batch)
    rc = torch.empty(batch, dtype=torch.float64, device="cuda")
    assert lib.hbem_lu_rcond(n, batch, P(Ar), P(Ai), n, n * n, P(anorm), P(rc), st) == 0
    return anorm.cpu().numpy(), rc.cpu().numpy()


@pytest.mark.parametrize("mode", [0, 1])
@pytest.mark.parametrize("n", [1, 7, 200, 1059])
def test_rcond_matches_lapack_cgecon(n, mode):
    """The reference's estimateReciprocalCondition: clange('1') + cgecon on cgetrf factors
    (with either solve scheme inside the estimator)."""
    from scipy.linalg import lapack

    A, _ = _lu_case(n, 2, 500 + n)
    # a badly scaled column makes the estimate non-trivial
    A[:, :, n // 2] *= 1e-3
    lib = load_library()
    assert lib.hbem_set_tuning(2, mode) == 0
    try:
        anorm, rc = _rcond_gpu(A)
    finally:
        lib.hbem_set_tuning(2, 0)
    for m in range(A.shape[0]):
        ref_norm = float(np.abs(A[m].astype(np.complex128)).sum(axis=0).max())
        assert abs(anorm[m] - ref_norm) <= 1e-5 * ref_norm
        lu, piv, info = lapack.cgetrf(A[m])
        ref, info2 = lapack.cgecon(lu, ref_norm, norm="1")
        assert info == 0 and info2 == 0
        assert abs(rc[m] - ref) <= 1e-2 * ref, (rc[m], ref)
        exact = 1.0 / (ref_norm * np.abs(np.linalg.inv(A[m].astype(np.complex128))).sum(axis=0).max())
        assert rc[m] >= exact * (1 - 1e-3)


def test_rcond_of_bem_matrix_matches_lapack():
    from scipy.linalg import lapack

    b = golden_buffers("horn_quarter")
    q = _q(b.n_triangles, 1)
    with _session("horn_quarter") as s:
        Ar, Ai, br, bi = s.assemble([30.0, 140.0], np.repeat(q[None, :], 2, axis=0))
        A = _host(Ar, Ai).astype(np.complex64)
    anorm, rc = _rcond_gpu(A)
    for m in range(2):
        ref_norm = float(np.abs(A[m].astype(np.complex128)).sum(axis=0).max())
        lu, piv, info = lapack.cgetrf(A[m])
        ref, _ = lapack.cgecon(lu, ref_norm, norm="1")
        assert abs(rc[m] - ref) <= 1e-2 * ref, (rc[m], ref)


def test_singular_pivot_reports_info():
    n = 8
    A = np.eye(n, dtype=np.complex64)
    A[3, 3] = 0.0
    A[3, :] = 0.0
    Ar, Ai = _dev(A[None])
    piv, info = _factor(Ar, Ai, n, 1)
    assert int(info[0]) == 4


def test_bem_matrix_solve_matches_lapack():
    b = golden_buffers("horn_quarter")
    q = _q(b.n_triangles, 1)
    with _session("horn_quarter") as s:
        Ar, Ai, br, bi = s.assemble([30.0], q[None, :])
        A = _host(Ar, Ai)[0]
        rhs = _host(br, bi)[0]
        n = s.n_dof
        piv, info = _factor(Ar, Ai, n, 1)
        Br, Bi = br[:, :, None].contiguous(), bi[:, :, None].contiguous()
        _solve(Ar, Ai, piv, Br, Bi, n, 1, 1)
    x = _host(Br, Bi)[0, :, 0]
    ref = dense_solve(A, rhs, "f64")
    assert rel(x, ref) < 1e-5


# ------------------------------------------------------------------ field / tags
@pytest.mark.parametrize("name", ["ico2", "horn_quarter", "yz_half", "xy_half"])
def test_field_matches_oracle(name):
    b = golden_buffers(name)
    o = Oracle(b, SYM[name], "f64")
    rng = np.random.default_rng(4)
    p = (rng.normal(size=b.p1_dof_count) + 1j * rng.normal(size=b.p1_dof_count)).astype(np.complex64)
    q = _q(b.n_triangles, 6)
    obs = rng.normal(size=(3, 29)) * 1.5 + np.array([[0.3], [0.2], [1.0]])
    ref = o.field(33.0, p, q, obs)
    with _session(name) as s:
        pr, pi = _dev(p[None])
        fr, fi = s.field([33.0], pr, pi, q[None], obs)
    assert rel(_host(fr, fi)[0], ref) < 1e-4


def test_tag_average_matches_oracle():
    b = golden_buffers("horn_quarter")
    o = Oracle(b, 3, "f64")
    rng = np.random.default_rng(8)
    p = (rng.normal(size=(2, b.p1_dof_count)) + 1j * rng.normal(size=(2, b.p1_dof_count))).astype(np.complex64)
    with _session("horn_quarter") as s:
        pr, pi = _dev(p)
        out = s.tag_average(pr, pi, [1, 2, 99]).cpu().numpy()
    for f in range(2):
        for j, tag in enumerate([1, 2, 99]):
            want = o.tag_average(p[f], tag)
            assert abs(complex(out[f, j, 0], out[f, j, 1]) - want) <= 1e-12 + 1e-9 * abs(want)


def _refine(A0r, A0i, LUr, LUi, piv, Br, Bi, Xr, Xi, n, batch, tol, max_iter):
    import ctypes

    lib = load_library()
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    iters = torch.zeros(batch, dtype=torch.int32, device="cuda")
    resid = torch.zeros(batch, dtype=torch.float64, device="cuda")
    P = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    rc = lib.hbem_refine(n, batch, P(A0r), P(A0i), n, n * n, P(LUr), P(LUi), n * n, P(piv), n, P(Br), P(Bi), n,
                         P(Xr), P(Xi), n, tol, max_iter, P(iters), P(resid), st)
    assert rc == 0
    return iters.cpu().numpy(), resid.cpu().numpy()


@pytest.mark.parametrize("n", [130, 700])
def test_mixed_precision_lu_with_refinement(n):
    """BF16x3 tensor-core trailing updates, then FP64-residual refinement to 1e-6."""
    batch = 2
    A, b = _lu_case(n, batch, 100 + n)
    A0r, A0i = _dev(A)
    LUr, LUi = A0r.clone(), A0i.clone()
    piv, info = _factor(LUr, LUi, n, batch, precision=1)
    assert int(info.abs().sum()) == 0
    Xr, Xi = _dev(b[:, :, None])
    _solve(LUr, LUi, piv, Xr, Xi, n, 1, batch)
    x0 = _host(Xr, Xi)[:, :, 0]
    Br, Bi = _dev(b)
    Xr2, Xi2 = Xr[:, :, 0].contiguous(), Xi[:, :, 0].contiguous()
    iters, resid = _refine(A0r, A0i, LUr, LUi, piv, Br, Bi, Xr2, Xi2, n, batch, 1e-6, 10)
    x = _host(Xr2, Xi2)
    for m in range(batch):
        ref = np.linalg.solve(A[m].astype(np.complex128), b[m].astype(np.complex128))
        assert rel(x0[m], ref) < 1e-3          # unrefined BF16x3 factors
        assert resid[m] <= 1e-6
        assert rel(x[m], ref) < 1e-5           # refined


@pytest.mark.parametrize("n,batch", [(1043, 4), (3300, 1)])
def test_mixed_lu_two_block_update_matches_one_block(n, batch):
    """The mixed LU's 128-column blocks (two-half swaps and TRSM, one K = 128 tensor-core update per block)
    against its 64-column blocks (K = 64): the same pivots where the FP32 panels see the same data up to
    BF16x3 rounding, residuals of the same size, and both refined to 1e-6 against LAPACK."""
    lib = load_library()
    A, b = _lu_case(n, batch, 300 + n)
    out = {}
    for blk in (64, 128):
        A0r, A0i = _dev(A)
        LUr, LUi = A0r.clone(), A0i.clone()
        assert lib.hbem_set_tuning(9, blk) == 0
        try:
            piv, info = _factor(LUr, LUi, n, batch, precision=1)
        finally:
            lib.hbem_set_tuning(9, 0)
        assert int(info.abs().sum()) == 0
        Xr, Xi = _dev(b[:, :, None])
        _solve(LUr, LUi, piv, Xr, Xi, n, 1, batch)
        x0 = _host(Xr, Xi)[:, :, 0]
        Br, Bi = _dev(b)
        Xr2, Xi2 = Xr[:, :, 0].contiguous(), Xi[:, :, 0].contiguous()
        iters, resid = _refine(A0r, A0i, LUr, LUi, piv, Br, Bi, Xr2, Xi2, n, batch, 1e-6, 10)
        out[blk] = (x0, _host(Xr2, Xi2), resid)
    for m in range(batch):
        ref = np.linalg.solve(A[m].astype(np.complex128), b[m].astype(np.complex128))
        e64, e128 = rel(out[64][0][m], ref), rel(out[128][0][m], ref)
        assert e128 < 1e-3 and e128 < 4 * e64 + 1e-6   # unrefined BF16x3 factors, either blocking
        assert out[128][2][m] <= 1e-6
        assert rel(out[128][1][m], ref) < 1e-5


def test_wavefront_wait_that_runs_out_reports_state_error_and_nan():
    """A wavefront-solve wait bounded to one poll (HBEM_TUNE_WAVE_SPIN = 1) gives up before the earlier block's
    x arrives: the launch aborts, the unfinished x is NaN, and hbem_solve_status reports HBEM_ERR_STATE once (the
    report clears it).  With the built-in limit the same solve is exact again: the context stays usable."""
    lib = load_library()
    n = 2048
    A, b = _lu_case(n, 1, 77)
    Ar, Ai = _dev(A)
    br, bi = _dev(b)
    piv = torch.empty((1, n), dtype=torch.int32, device="cuda")
    info = torch.empty(1, dtype=torch.int32, device="cuda")
    assert lib.hbem_lu_factor(n, 1, _t_ptr(Ar), _t_ptr(Ai), n, n * n, _t_ptr(piv), n, _t_ptr(info), 0, None) == 0
    try:
        assert lib.hbem_set_tuning(HBEM_TUNE_LU_SOLVE, 3) == 0
        assert lib.hbem_set_tuning(HBEM_TUNE_WAVE_SPIN, 1) == 0
        xr, xi = br.clone(), bi.clone()
        assert lib.hbem_lu_solve(n, 1, 1, _t_ptr(Ar), _t_ptr(Ai), n, n * n, _t_ptr(piv), n, _t_ptr(xr), _t_ptr(xi),
                                 1, n, HBEM_TRANS_N, None) == 0
        assert lib.hbem_solve_status(None) == HBEM_ERR_STATE
        assert "timed out" in last_error(lib)
        assert torch.isnan(xr).any()
        assert lib.hbem_solve_status(None) == 0   # reported once
    finally:
        lib.hbem_set_tuning(HBEM_TUNE_WAVE_SPIN, 0)
        lib.hbem_set_tuning(HBEM_TUNE_LU_SOLVE, 0)
    xr, xi = br.clone(), bi.clone()
    assert lib.hbem_lu_solve(n, 1, 1, _t_ptr(Ar), _t_ptr(Ai), n, n * n, _t_ptr(piv), n, _t_ptr(xr), _t_ptr(xi), 1, n,
                             HBEM_TRANS_N, None) == 0
    assert lib.hbem_solve_status(None) == 0
    x = _host(xr, xi)[0]
    ref = np.linalg.solve(A[0].astype(np.complex128), b[0].astype(np.complex128))
    assert rel(x, ref) < 1e-4


@pytest.mark.parametrize("name", ["ico2", "yzxz_quarter", "xy_half"])
def test_assemble_multi_equals_one_pass_per_source(name):
    """hbem_assemble_multi: one pass for 3 sources gives the matrix of a single-source pass and each source's
    right-hand side as its own pass gives it (FP32 atomics reorder sums: 1e-6)."""
    b = golden_buffers(name)
    T, n = b.n_triangles, b.p1_dof_count
    ks = [18.3, 91.6]
    qs = np.stack([np.stack([_q(T, 10 * s + f) for f in range(2)]) for s in range(3)])   # (S, F, T)
    qs[1, :, ::3] = 0.0   # sources with different supports
    lib = load_library()
    with _session(name) as s:
        Ar, Ai, br1, bi1 = s.assemble(ks, qs[0])
        refs = [_host(*s.assemble(ks, qs[k])[2:]) for k in range(3)]
        qr = torch.tensor(np.ascontiguousarray(qs.real, np.float32), device="cuda")
        qi = torch.tensor(np.ascontiguousarray(qs.imag, np.float32), device="cuda")
        Mr, Mi = torch.empty_like(Ar), torch.empty_like(Ai)
        Br = torch.empty((3, 2, n), dtype=torch.float32, device="cuda")
        Bi = torch.empty_like(Br)
        k_arr = np.asarray(ks, np.float32)
        rc = lib.hbem_assemble_multi(s.handle, 2, k_arr.ctypes.data_as(ctypes.c_void_p), None, 3, _t_ptr(qr),
                                     _t_ptr(qi), T, 2 * T, None, None, _t_ptr(Mr), _t_ptr(Mi), n, n * n, _t_ptr(Br),
                                     _t_ptr(Bi), n, 2 * n, 7, None)
        assert rc == 0, last_error(lib)
        torch.cuda.synchronize()
    A = _host(Ar, Ai)
    assert rel(_host(Mr, Mi), A) < 1e-6
    B = _host(Br, Bi)
    for k in range(3):   # (a one-triangle mesh leaves the zeroed source with b = 0 exactly)
        assert np.linalg.norm(B[k] - refs[k]) <= 1e-6 * max(np.linalg.norm(refs[k]), 1e-30)


@pytest.mark.parametrize("name,level,threshold", [("near", 2, 1.5), ("ico2", 1, 1.5), ("horn_quarter", 2, 1.5),
                                                  ("horn_quarter", 1, 1.0), ("ico2", 2, 2.5)])
def test_near_quadrature_assembly_matches_oracle(name, level, threshold):
    """Near-field subdivision on the GPU (hbem_session_set_near_quadrature) against the oracle's restatement of
    the reference's CPU correction (main.swift:3072-3202): the same near pairs, and the corrected matrix and
    right-hand side with the near corrections within 1e-4."""
    b = golden_buffers(name)
    o = Oracle(b, SYM[name], "f64")
    q = _q(b.n_triangles, 8)
    k = 18.3
    A_ref, b_ref = o.corrected(k, q)
    n_ref = o.near_correct(A_ref, b_ref, k, q, level=level, threshold=threshold)
    with NativeSession(b, symmetry_plane={0: None, 1: "yz", 3: "yz+xz", 4: "xy"}[SYM[name]],
                       check_open_edges=False, near_quadrature=(level, threshold)) as s:
        assert s.query("near_pairs") == n_ref == len(o.near_pairs(threshold))
        assert s.near_quadrature["pair_count"] == n_ref
        Ar, Ai, br, bi = s.assemble([k], q[None, :])
    assert n_ref > 0
    assert rel(_host(Ar, Ai)[0], A_ref) < 1e-4
    assert rel(_host(br, bi)[0], b_ref) < 1e-4


def test_near_quadrature_on_the_reference_fixture_and_off_again():
    """The reference's test on the GPU path: level 2 at threshold 1.5 moves the near fixture's (0, 1) block
    towards the level-4 subdivided helper (golden); level 0 restores the plain corrected matrix exactly."""
    from conftest import golden

    b = golden_buffers("near")
    q = np.array([1.0, 0.0], np.complex64)
    k = 1.8318326
    with NativeSession(b, check_open_edges=False) as s:
        A0 = _host(*s.assemble([k], q[None, :])[:2])[0]
        lib = load_library()
        assert lib.hbem_session_set_near_quadrature(s.handle, 2, 1.5) == 0
        A1 = _host(*s.assemble([k], q[None, :])[:2])[0]
        assert lib.hbem_session_set_near_quadrature(s.handle, 0, 0.0) == 0
        assert s.query("near_pairs") == 0
        A2 = _host(*s.assemble([k], q[None, :])[:2])[0]
        assert lib.hbem_session_set_near_quadrature(s.handle, 3, 1.5) == -1
        assert lib.hbem_session_set_near_quadrature(s.handle, 1, -1.0) == -1
    ref = golden("pair_blocks.npz")["0__dlp"]
    blk = np.ix_([0, 1, 2], [3, 4, 5])
    assert np.linalg.norm(A1[blk] - ref) < 0.1 * np.linalg.norm(A0[blk] - ref)
    assert rel(A2, A0) < 1e-6
