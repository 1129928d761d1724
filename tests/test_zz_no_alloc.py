"""hbem_refine_noalloc against hbem_refine, through the C ABI.

The no-allocation entry keeps its scratch in one fixed device array shared
by every call.  Two calls in a row must each give what hbem_refine gives on
the same inputs (the second call starts from the first call's leftover
scratch).  Tolerance: both refine to ||b - A x|| / ||b|| <= 1e-6, so their
solutions agree within 1e-5 relative L2, the refinement tests' bound.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover - CPU containers
    pytest.skip("needs a CUDA device", allow_module_level=True)

from hornlab_metal_bem_b200.native import last_error, load_library  # noqa: E402

HBEM_ERR_ARG = -1


def _p(t):
    return ctypes.c_void_p(t.data_ptr())


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _case(n, batch, seed):
    rng = np.random.default_rng(seed)
    A = rng.normal(size=(batch, n, n)) + 1j * rng.normal(size=(batch, n, n))
    A += np.eye(n)[None] * (2.0 * np.sqrt(n))
    b = rng.normal(size=(batch, n)) + 1j * rng.normal(size=(batch, n))
    return A.astype(np.complex64), b.astype(np.complex64)


def _dev(z):
    return (torch.from_numpy(np.ascontiguousarray(z.real, np.float32)).cuda(),
            torch.from_numpy(np.ascontiguousarray(z.imag, np.float32)).cuda())


def _host(re, im):
    return re.cpu().numpy().astype(np.float64) + 1j * im.cpu().numpy().astype(np.float64)


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _factor_and_first_solve(lib, A, b, n, batch):
    """Tensor-core (mixed) factors, so that refinement has passes to make."""
    A0r, A0i = _dev(A)
    LUr, LUi = A0r.clone(), A0i.clone()
    piv = torch.zeros((batch, n), dtype=torch.int32, device="cuda")
    info = torch.zeros(batch, dtype=torch.int32, device="cuda")
    assert lib.hbem_lu_factor(n, batch, _p(LUr), _p(LUi), n, n * n, _p(piv), n, _p(info), 1, _stream()) == 0
    assert int(info.abs().sum()) == 0
    Br, Bi = _dev(b)
    Xr, Xi = Br.clone(), Bi.clone()
    assert lib.hbem_lu_solve(n, 1, batch, _p(LUr), _p(LUi), n, n * n, _p(piv), n, _p(Xr), _p(Xi), 1, n, 0,
                             _stream()) == 0
    return A0r, A0i, LUr, LUi, piv, Br, Bi, Xr, Xi


def _refine(lib, entry, n, batch, case, Xr, Xi):
    A0r, A0i, LUr, LUi, piv, Br, Bi = case
    iters = torch.zeros(batch, dtype=torch.int32, device="cuda")
    resid = torch.zeros(batch, dtype=torch.float64, device="cuda")
    rc = getattr(lib, entry)(n, batch, _p(A0r), _p(A0i), n, n * n, _p(LUr), _p(LUi), n * n, _p(piv), n, _p(Br), _p(Bi),
                             n, _p(Xr), _p(Xi), n, 1e-6, 10, _p(iters), _p(resid), _stream())
    assert rc == 0, last_error(lib)
    torch.cuda.synchronize()
    return iters.cpu().numpy(), resid.cpu().numpy()


def test_noalloc_refine_matches_refine_twice_in_a_row():
    lib = load_library()
    for n, batch, seed in [(700, 3, 41), (257, 2, 42)]:
        A, b = _case(n, batch, seed)
        A0r, A0i, LUr, LUi, piv, Br, Bi, Xr, Xi = _factor_and_first_solve(lib, A, b, n, batch)
        case = (A0r, A0i, LUr, LUi, piv, Br, Bi)
        Xr_a, Xi_a = Xr.clone(), Xi.clone()
        it_a, res_a = _refine(lib, "hbem_refine", n, batch, case, Xr_a, Xi_a)
        Xr_b, Xi_b = Xr.clone(), Xi.clone()
        it_b, res_b = _refine(lib, "hbem_refine_noalloc", n, batch, case, Xr_b, Xi_b)
        xa, xb = _host(Xr_a, Xi_a), _host(Xr_b, Xi_b)
        for m in range(batch):
            assert res_b[m] <= 1e-6
            assert _rel(xb[m], xa[m]) < 1e-5
            ref = np.linalg.solve(A[m].astype(np.complex128), b[m].astype(np.complex128))
            assert _rel(xb[m], ref) < 1e-5
        assert np.all(it_b >= 1)


def test_noalloc_refine_rejects_sizes_beyond_its_scratch():
    lib = load_library()
    t = torch.zeros(8, dtype=torch.float32, device="cuda")
    piv = torch.zeros(8, dtype=torch.int32, device="cuda")
    args = lambda n, batch, stride: (n, batch, _p(t), _p(t), n, n * n, _p(t), _p(t), n * n, _p(piv), n,  # noqa: E731
                                     _p(t), _p(t), stride, _p(t), _p(t), stride, 1e-6, 10, None, None, _stream())
    assert lib.hbem_refine_noalloc(*args(2, 257, 2)) == HBEM_ERR_ARG
    assert "scratch limit" in last_error(lib)
    assert lib.hbem_refine_noalloc(*args(2, 2, 1 << 19)) == HBEM_ERR_ARG
    assert "scratch limit" in last_error(lib)


_POOL_USED_CURRENT, _POOL_USED_HIGH = 7, 8   # cudaMemPoolAttrUsedMemCurrent / cudaMemPoolAttrUsedMemHigh


def _pool():
    """The device's default stream-ordered pool, queried through the CUDA runtime the library loaded."""
    rt = ctypes.CDLL("libcudart.so.12")
    pool = ctypes.c_void_p()
    assert rt.cudaDeviceGetDefaultMemPool(ctypes.byref(pool), torch.cuda.current_device()) == 0
    return rt, pool


def _pool_attr(rt, pool, attr):
    v = ctypes.c_uint64()
    assert rt.cudaMemPoolGetAttribute(pool, attr, ctypes.byref(v)) == 0
    return v.value


def _pool_reset_high(rt, pool):
    zero = ctypes.c_uint64(0)
    assert rt.cudaMemPoolSetAttribute(pool, _POOL_USED_HIGH, ctypes.byref(zero)) == 0


def test_noalloc_refine_takes_nothing_from_the_stream_ordered_pool():
    """The point of the entry: no device allocation on any path it takes.  Around each call, the default pool's
    high-water mark of memory in use is reset and must not rise above what was in use before, for every
    triangular-solve variant (HBEM_TUNE_LU_SOLVE 0..3) of its correction solves.  hbem_refine, which takes its
    scratch from that pool, raises the mark: the measurement sees allocations."""
    lib = load_library()
    n, batch = 300, 2
    A, b = _case(n, batch, 43)
    A0r, A0i, LUr, LUi, piv, Br, Bi, Xr, Xi = _factor_and_first_solve(lib, A, b, n, batch)
    case = (A0r, A0i, LUr, LUi, piv, Br, Bi)
    rt, pool = _pool()
    ref = [np.linalg.solve(A[m].astype(np.complex128), b[m].astype(np.complex128)) for m in range(batch)]
    try:
        for mode in (0, 1, 2, 3):
            assert lib.hbem_set_tuning(2, mode) == 0
            X2r, X2i = Xr.clone(), Xi.clone()
            torch.cuda.synchronize()
            before = _pool_attr(rt, pool, _POOL_USED_CURRENT)
            _pool_reset_high(rt, pool)
            _refine(lib, "hbem_refine_noalloc", n, batch, case, X2r, X2i)
            assert _pool_attr(rt, pool, _POOL_USED_HIGH) <= before, mode
            x = _host(X2r, X2i)
            for m in range(batch):
                assert _rel(x[m], ref[m]) < 1e-5
        # control: the allocating twin shows up in the same measurement
        X3r, X3i = Xr.clone(), Xi.clone()
        torch.cuda.synchronize()
        before = _pool_attr(rt, pool, _POOL_USED_CURRENT)
        _pool_reset_high(rt, pool)
        _refine(lib, "hbem_refine", n, batch, case, X3r, X3i)
        assert _pool_attr(rt, pool, _POOL_USED_HIGH) > before
    finally:
        lib.hbem_set_tuning(2, 0)
