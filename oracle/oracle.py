"""TEST INFRASTRUCTURE — Python face of the CPU oracle (``hbem_oracle.c``).

Only tests/, ``__graft_entry__.smoke()`` and ``bench.py`` (its cpu_baseline and
``--impl reference`` arms) import this module, as the checker or as the timed
CPU baseline.  The product path never does.

It wraps the C restatement of the reference's CPU path (see the header of
``hbem_oracle.c`` for the file:line map) and adds the dense solve the
reference delegates to Apple Accelerate ``cgesv`` (``main.swift:7834-7941``);
the stand-in here is LAPACK ``cgesv``/``zgesv`` from SciPy (OpenBLAS).
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
BUILD = HERE / "_build"


class _Geom(ctypes.Structure):
    _fields_ = [
        ("n_vertices", ctypes.c_int),
        ("n_triangles", ctypes.c_int),
        ("n_dof", ctypes.c_int),
        ("sym", ctypes.c_int),
        ("verts", ctypes.c_void_p),
        ("tris", ctypes.c_void_p),
        ("l2g", ctypes.c_void_p),
        ("areas", ctypes.c_void_p),
        ("normals", ctypes.c_void_p),
    ]


def build() -> None:
    """Compile the oracle libraries (gcc + OpenMP) into ``oracle/_build``."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


def _lib(precision: str):
    name = {"f32": "libhbem_oracle_f32.so", "f64": "libhbem_oracle_f64.so", "g64": "libhbem_oracle_g64.so"}[precision]
    path = BUILD / name
    if not path.exists():
        build()
    return ctypes.CDLL(str(path))


def _ptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


class Oracle:
    """CPU oracle bound to one geometry (``GeometryBuffers``-like object)."""

    def __init__(self, buffers, symmetry_code: int = 0, precision: str = "f64", threads: int | None = None,
                 vertices_3xv=None):
        """precision: "f32" (the reference's arithmetic), "f64", or "g64" (f64 with float64 geometry:
        ``vertices_3xv`` (3, V) float64 replaces the buffers' vertices, areas and normals are rebuilt
        in float64 -- the finite-difference reference for shape gradients)."""
        self.precision = precision
        self.lib = _lib(precision)
        self.pre = {"f32": "og32_", "f64": "og64_", "g64": "og64g_"}[precision]
        self.real = np.float32 if precision == "f32" else np.float64
        self._ct = ctypes.c_float if precision == "f32" else ctypes.c_double
        tris = np.ascontiguousarray(buffers.triangles_3xm_i32, dtype=np.int32)
        if precision == "g64":
            v = np.asarray(buffers.vertices_3xn_f32 if vertices_3xv is None else vertices_3xv, dtype=np.float64)
            p0, p1, p2 = (v[:, tris[i]].T for i in range(3))
            cross = np.cross(p1 - p0, p2 - p0)
            twice = np.linalg.norm(cross, axis=1)
            geo = [np.ascontiguousarray(v), np.ascontiguousarray(0.5 * twice),
                   np.ascontiguousarray((cross / twice[:, None]).T)]
        else:
            geo = [np.ascontiguousarray(buffers.vertices_3xn_f32, dtype=np.float32),
                   np.ascontiguousarray(buffers.triangle_areas_f32, dtype=np.float32),
                   np.ascontiguousarray(buffers.triangle_normals_3xm_f32, dtype=np.float32)]
        self._keep = [geo[0], tris, np.ascontiguousarray(buffers.p1_local2global_i32, dtype=np.int32), geo[1], geo[2]]
        self.tags = np.ascontiguousarray(buffers.physical_tags_i32, dtype=np.int32)
        self.n = int(buffers.p1_dof_count)
        self.T = int(buffers.triangles_3xm_i32.shape[1])
        self.geom = _Geom(
            int(buffers.vertices_3xn_f32.shape[1]), self.T, self.n, int(symmetry_code),
            *[_ptr(a) for a in self._keep],
        )
        self.set_threads(threads if threads is not None else len(os.sched_getaffinity(0)))

    def _fn(self, name):
        return getattr(self.lib, self.pre + name)

    def set_threads(self, n: int) -> int:
        return int(self._fn("set_threads")(ctypes.c_int(int(n))))

    # -- assembly -----------------------------------------------------------
    def _split(self, z, n):
        if z is None:
            return None, None
        z = np.asarray(z, dtype=np.complex128).reshape(n)
        return (np.ascontiguousarray(z.real, dtype=np.float32), np.ascontiguousarray(z.imag, dtype=np.float32))

    def regular(self, k: float, q=None, k_imag: float = 0.0, beta=None):
        n = self.n
        Are = np.zeros((n, n), self.real); Aim = np.zeros((n, n), self.real)
        bre = np.zeros(n, self.real); bim = np.zeros(n, self.real)
        qre, qim = self._split(q, self.T)
        brr, bri = self._split(beta, self.T)
        self._fn("regular_assemble")(
            ctypes.byref(self.geom), self._ct(k), self._ct(k_imag), _ptr(qre), _ptr(qim), _ptr(brr), _ptr(bri),
            _ptr(Are), _ptr(Aim), _ptr(bre), _ptr(bim),
        )
        return Are + 1j * Aim, bre + 1j * bim

    def duffy_correct(self, A, b, k: float, q=None, k_imag: float = 0.0, beta=None, order: int = 4) -> int:
        """Add the Duffy singular corrections to ``A``/``b`` in place; returns unique triplets.  ``order``:
        Gauss-Legendre points per Duffy coordinate (the reference's rule has 4)."""
        Are = np.ascontiguousarray(A.real, dtype=self.real); Aim = np.ascontiguousarray(A.imag, dtype=self.real)
        bre = np.ascontiguousarray(b.real, dtype=self.real); bim = np.ascontiguousarray(b.imag, dtype=self.real)
        qre, qim = self._split(q, self.T)
        brr, bri = self._split(beta, self.T)
        args = (ctypes.byref(self.geom), self._ct(k), self._ct(k_imag), _ptr(qre), _ptr(qim), _ptr(brr), _ptr(bri),
                _ptr(Are), _ptr(Aim), _ptr(bre), _ptr(bim))
        u = (self._fn("duffy_correct")(*args) if order == 4
             else self._fn("duffy_correct_m")(*args, ctypes.c_int(int(order))))
        A[...] = Are + 1j * Aim
        b[...] = bre + 1j * bim
        return int(u)

    def near_pairs(self, threshold: float = 1.5):
        """Near, non-touching (test, trial, test_mask, trial_mask) pairs of the near-field option."""
        npairs = self._fn("near_pairs")(ctypes.byref(self.geom), ctypes.c_double(threshold), None, 0)
        out = np.zeros((max(npairs, 1), 4), np.int32)
        self._fn("near_pairs")(ctypes.byref(self.geom), ctypes.c_double(threshold), _ptr(out), ctypes.c_int(npairs))
        return out[:npairs]

    def near_correct(self, A, b, k: float, q=None, k_imag: float = 0.0, beta=None, level: int = 2,
                     threshold: float = 1.5) -> int:
        """Add the near-field subdivision corrections (subdivided - regular blocks of near, non-touching
        pairs, the reference's optional near quadrature) to ``A``/``b`` in place; returns the pair count."""
        Are = np.ascontiguousarray(A.real, dtype=self.real); Aim = np.ascontiguousarray(A.imag, dtype=self.real)
        bre = np.ascontiguousarray(b.real, dtype=self.real); bim = np.ascontiguousarray(b.imag, dtype=self.real)
        qre, qim = self._split(q, self.T)
        brr, bri = self._split(beta, self.T)
        npairs = self._fn("near_correct")(
            ctypes.byref(self.geom), self._ct(k), self._ct(k_imag), _ptr(qre), _ptr(qim), _ptr(brr), _ptr(bri),
            _ptr(Are), _ptr(Aim), _ptr(bre), _ptr(bim), ctypes.c_int(int(level)), ctypes.c_double(threshold))
        A[...] = Are + 1j * Aim
        b[...] = bre + 1j * bim
        return int(npairs)

    def corrected(self, k: float, q=None, k_imag: float = 0.0, beta=None, duffy_order: int = 4):
        """Regular 6x6 assembly plus Duffy corrections: the reference's 'corrected' mode (``duffy_order`` 4);
        other orders give the convergence study of its singular quadrature."""
        A, b = self.regular(k, q, k_imag, beta)
        self.duffy_correct(A, b, k, q, k_imag, beta, order=duffy_order)
        return A, b

    def duffy_pairs(self):
        counts = (ctypes.c_int * 3)()
        np_ = self._fn("duffy_pairs")(ctypes.byref(self.geom), None, 0, counts)
        pairs = np.zeros((max(np_, 1), 9), dtype=np.int32)
        self._fn("duffy_pairs")(ctypes.byref(self.geom), _ptr(pairs), ctypes.c_int(np_), counts)
        return pairs[:np_], {"coincident": counts[0], "edge": counts[1], "vertex": counts[2]}

    def unique_triplets(self, pairs) -> int:
        pairs = np.ascontiguousarray(pairs, dtype=np.int32)
        return int(self._fn("duffy_unique_triplets")(ctypes.byref(self.geom), _ptr(pairs), ctypes.c_int(pairs.shape[0])))

    def pair_blocks(self, test, trial, test_mask=0, trial_mask=0, mode=0, kind=0, locals_=None, level=0, k=1.0, k_imag=0.0):
        out = np.zeros(24, self.real)
        loc = None if locals_ is None else np.ascontiguousarray(locals_, dtype=np.int32)
        self._fn("pair_blocks")(
            ctypes.byref(self.geom), test, trial, test_mask, trial_mask, mode, kind, _ptr(loc), level,
            self._ct(k), self._ct(k_imag), _ptr(out),
        )
        slp = out[0:6:2] + 1j * out[1:6:2]
        dlp = (out[6::2] + 1j * out[7::2]).reshape(3, 3)
        return slp, dlp

    def rule(self, kind: int):
        rec = np.zeros((1536, 5), self.real)
        n = self._fn("duffy_rule_table")(ctypes.c_int(kind), _ptr(rec))
        return rec[:n]

    # -- field / reductions -------------------------------------------------
    def field(self, k: float, p, q, obs_3xn):
        obs = np.ascontiguousarray(obs_3xn, dtype=np.float32)
        nobs = obs.shape[1]
        p = np.asarray(p).reshape(self.n); q = np.asarray(q).reshape(self.T)
        pre = np.ascontiguousarray(p.real, self.real); pim = np.ascontiguousarray(p.imag, self.real)
        qre = np.ascontiguousarray(q.real, self.real); qim = np.ascontiguousarray(q.imag, self.real)
        ore = np.zeros(nobs, self.real); oim = np.zeros(nobs, self.real)
        self._fn("field")(
            ctypes.byref(self.geom), self._ct(k), _ptr(pre), _ptr(pim), _ptr(qre), _ptr(qim), _ptr(obs),
            ctypes.c_int(nobs), _ptr(ore), _ptr(oim),
        )
        return ore + 1j * oim

    def chief_rows(self, pts_3xm, k: float, q=None, k_imag: float = 0.0, beta=None):
        """CHIEF collocation rows at interior points (main.swift:1897-2036): (C (m, n), d (m,), ||C||_inf)
        with C p = d the vanishing exterior representation, Robin folded in as in the boundary rows."""
        pts = np.ascontiguousarray(pts_3xm, dtype=np.float32)
        m, n = pts.shape[1], self.n
        cre = np.zeros((m, n), self.real); cim = np.zeros((m, n), self.real)
        dre = np.zeros(m, self.real); dim = np.zeros(m, self.real)
        qre, qim = (None, None)
        if q is not None:
            qz = np.asarray(q, dtype=np.complex128).reshape(self.T)
            qre, qim = np.ascontiguousarray(qz.real, self.real), np.ascontiguousarray(qz.imag, self.real)
        brr = bri = None
        if beta is not None:
            bz = np.asarray(beta, dtype=np.complex128).reshape(self.T)
            brr, bri = np.ascontiguousarray(bz.real, self.real), np.ascontiguousarray(bz.imag, self.real)
        fn = self._fn("chief_rows")
        fn.restype = ctypes.c_double
        cn = fn(ctypes.byref(self.geom), _ptr(pts), ctypes.c_int(m), self._ct(k), self._ct(k_imag), _ptr(brr),
                _ptr(bri), _ptr(qre), _ptr(qim), _ptr(cre), _ptr(cim), _ptr(dre), _ptr(dim))
        return cre + 1j * cim, dre + 1j * dim, float(cn)

    def tag_average(self, p, tag: int) -> complex:
        p = np.asarray(p).reshape(self.n)
        pre = np.ascontiguousarray(p.real, self.real); pim = np.ascontiguousarray(p.imag, self.real)
        out = np.zeros(3, np.float64)
        self._fn("tag_average")(ctypes.byref(self.geom), _ptr(self.tags), _ptr(pre), _ptr(pim), ctypes.c_int(int(tag)), _ptr(out))
        return complex(out[0], out[1])


    # -- coupled infinite baffle ---------------------------------------------
    def aperture_triangles(self, tag: int):
        return np.flatnonzero(self.tags == int(tag)).astype(np.int32)

    def aperture_slp(self, ap, k: float, k_imag: float = 0.0):
        ap = np.ascontiguousarray(ap, dtype=np.int32)
        m = ap.shape[0]
        Sre = np.zeros((self.n, m), self.real); Sim = np.zeros((self.n, m), self.real)
        self._fn("aperture_slp")(ctypes.byref(self.geom), _ptr(ap), ctypes.c_int(m), self._ct(k), self._ct(k_imag),
                                 _ptr(Sre), _ptr(Sim))
        return Sre + 1j * Sim

    def aperture_avg(self, ap, k: float):
        ap = np.ascontiguousarray(ap, dtype=np.int32)
        m = ap.shape[0]
        Sre = np.zeros((m, m), self.real); Sim = np.zeros((m, m), self.real)
        self._fn("aperture_avg")(ctypes.byref(self.geom), _ptr(ap), ctypes.c_int(m), self._ct(k), _ptr(Sre), _ptr(Sim))
        return Sre + 1j * Sim

    def rayleigh(self, ap, k: float, qa, obs_3xn):
        ap = np.ascontiguousarray(ap, dtype=np.int32)
        obs = np.ascontiguousarray(obs_3xn, dtype=np.float32)
        qa = np.asarray(qa)
        qre = np.ascontiguousarray(qa.real, self.real); qim = np.ascontiguousarray(qa.imag, self.real)
        ore = np.zeros(obs.shape[1], self.real); oim = np.zeros(obs.shape[1], self.real)
        self._fn("rayleigh")(ctypes.byref(self.geom), _ptr(ap), ctypes.c_int(ap.shape[0]), self._ct(k), _ptr(qre),
                             _ptr(qim), _ptr(obs), ctypes.c_int(obs.shape[1]), _ptr(ore), _ptr(oim))
        return ore + 1j * oim

    def coupled_ib_solve(self, A, b, ap, k: float, field_k: float, k_imag: float = 0.0, precision: str = "f64"):
        """Augmented system [[A, -S_ia], [P_avg, -2 S_aa]] [p; q_a] = [b; 0] (main.swift:7504-7595)."""
        S_ia = self.aperture_slp(ap, k, k_imag)
        S_aa = self.aperture_avg(ap, field_k)
        n, m = self.n, len(ap)
        l2g = np.asarray(self._keep[2])
        P = np.zeros((m, n))
        for r, t in enumerate(ap):
            for d in l2g[t]:
                P[r, d] += 1.0 / 3.0
        Aug = np.zeros((n + m, n + m), np.complex128)
        Aug[:n, :n] = A
        Aug[:n, n:] = -S_ia
        Aug[n:, :n] = P
        Aug[n:, n:] = -2.0 * S_aa
        rhs = np.concatenate([np.asarray(b, np.complex128), np.zeros(m)])
        x = dense_solve(Aug, rhs, precision)
        return x[:n], x[n:], S_ia, S_aa


def dense_solve(A, b, precision: str = "f32"):
    """LAPACK ``cgesv`` (complex64) or ``zgesv`` (complex128): the Accelerate stand-in."""
    from scipy.linalg import lapack

    if precision == "f32":
        lu, piv, x, info = lapack.cgesv(np.asarray(A, np.complex64), np.asarray(b, np.complex64))
    else:
        lu, piv, x, info = lapack.zgesv(np.asarray(A, np.complex128), np.asarray(b, np.complex128))
    if info != 0:
        raise RuntimeError(f"LAPACK gesv info={info}")
    return x


def chief_lstsq(A, b, C, d, weight: float = 1.0):
    """The reference's CHIEF least squares (main.swift:7186-7409): minimise ||[A; s C] p - [b; s d]||_2 in
    complex128 (LAPACK zgels), s = weight ||A||_inf / ||C||_inf (largest row sums of |a|, |c|).  b and d may
    hold several right-hand sides as columns.  Returns (p, s, per-column ||s (C p - d)|| / ||b||)."""
    from scipy.linalg import lapack

    A = np.asarray(A, np.complex128); C = np.asarray(C, np.complex128)
    b = np.asarray(b, np.complex128); d = np.asarray(d, np.complex128)
    one = b.ndim == 1
    B, D = (b[:, None], d[:, None]) if one else (b, d)
    an = float(np.abs(A).sum(axis=1).max())
    cn = float(np.abs(C).sum(axis=1).max())
    s = weight * (an / cn if cn > 0 else 1.0)
    M = np.vstack([A, s * C])
    R = np.vstack([B, s * D])
    _, x, info = lapack.zgels(M, R)
    if info != 0:
        raise RuntimeError(f"LAPACK zgels info={info}")
    p = x[:A.shape[1]]
    res = np.linalg.norm(s * (C @ p - D), axis=0) / np.where(np.linalg.norm(B, axis=0) > 0,
                                                            np.linalg.norm(B, axis=0), 1.0)
    return (p[:, 0] if one else p), s, (float(res[0]) if one else res)


def solve_case(oracle: Oracle, k: float, q, obs_3xn, precision: str = "f32"):
    """One frequency of the reference's corrected path: assemble, solve, field."""
    A, b = oracle.corrected(k, q)
    p = dense_solve(A, b, precision)
    field = oracle.field(k, p, q, obs_3xn)
    return A, b, p, field
