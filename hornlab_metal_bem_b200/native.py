"""ctypes binding of ``libhbem.so`` and the session object of the B200 path.

``NativeSession`` stands where the reference's ``MetalNativeStandardSession``
stands (``hornlab_metal_bem/metal/native.py:233-1203``): it owns one mesh's
resident geometry on the GPU and runs the batched
assemble -> LU -> solve -> field -> reductions operation.  Instead of a helper
subprocess with JSON manifests and float32 files, every call goes through the
C ABI declared in ``include/hbem.h``.

There is no CPU fallback: if the library is missing or no CUDA device is
visible, construction raises ``BackendUnavailable``.
"""
from __future__ import annotations

import ctypes
import math
import os
import time
from dataclasses import dataclass, field
from pathlib import Path
from typing import Any

import numpy as np

from .config import SYMMETRY_CODES
from .geometry import (
    GeometryBuffers,
    validate_native_infinite_baffle_aperture,
    validate_native_symmetry_plane,
)

LIB_PATH = Path(__file__).resolve().parent / "libhbem.so"

HBEM_OK = 0
HBEM_ASM_REGULAR = 1
HBEM_ASM_DUFFY = 2
HBEM_ASM_ZERO = 4
HBEM_ASM_CORRECTED = 7
HBEM_PREC_PLAIN = 0
HBEM_PREC_MIXED = 1
HBEM_PREC_FP64 = 2
HBEM_PREC_TF32X3 = 3
HBEM_TRANS_N, HBEM_TRANS_T, HBEM_TRANS_C = 0, 1, 2
# aperture faces from which the coupled solve uses the augmented (m + n) system
AUGMENTED_MIN_APERTURE = 512
QUERY_KEYS = {
    "n_dof": 0, "n_triangles": 1, "n_pairs": 2, "coincident": 3, "edge": 4, "vertex": 5,
    "image_pairs": 6, "unique_triplets": 7, "symmetry": 8, "kernel_launches": 9,
    "regular_evals": 10, "duffy_evals": 11, "aperture_triangles": 12, "near_pairs": 13,
}


class BackendUnavailable(RuntimeError):
    """The CUDA library or device needed by the B200 path is not available."""


# Drop-in alias for the reference's exception name (hornlab_metal_bem/backends.py).
AssemblyBackendUnavailable = BackendUnavailable

_c_int, _c_ll, _c_d, _vp = ctypes.c_int, ctypes.c_longlong, ctypes.c_double, ctypes.c_void_p
_SIGNATURES = {
    "hbem_version": ([], _c_int),
    "hbem_last_error": ([ctypes.c_char_p, ctypes.c_size_t], _c_int),
    "hbem_launch_count": ([], _c_ll),
    "hbem_session_create": ([_vp, _c_int, _vp, _c_int, _vp, _c_int, _vp, _vp, _vp, _c_int, _c_int,
                             ctypes.POINTER(_vp)], _c_int),
    "hbem_session_destroy": ([_vp], _c_int),
    "hbem_session_query": ([_vp, _c_int, ctypes.POINTER(_c_ll)], _c_int),
    "hbem_assemble": ([_vp, _c_int, _vp, _vp, _vp, _vp, _c_ll, _vp, _vp, _vp, _vp, _c_ll, _c_ll, _vp, _vp, _c_ll,
                       _c_int, _vp], _c_int),
    "hbem_lu_factor": ([_c_int, _c_int, _vp, _vp, _c_ll, _c_ll, _vp, _c_ll, _vp, _c_int, _vp], _c_int),
    "hbem_lu_solve": ([_c_int, _c_int, _c_int, _vp, _vp, _c_ll, _c_ll, _vp, _c_ll, _vp, _vp, _c_ll, _c_ll, _c_int,
                       _vp], _c_int),
    "hbem_refine": ([_c_int, _c_int, _vp, _vp, _c_ll, _c_ll, _vp, _vp, _c_ll, _vp, _c_ll, _vp, _vp, _c_ll, _vp, _vp,
                     _c_ll, _c_d, _c_int, _vp, _vp, _vp], _c_int),
    "hbem_refine_noalloc": ([_c_int, _c_int, _vp, _vp, _c_ll, _c_ll, _vp, _vp, _c_ll, _vp, _c_ll, _vp, _vp, _c_ll, _vp,
                             _vp, _c_ll, _c_d, _c_int, _vp, _vp, _vp], _c_int),
    "hbem_chief_lstsq": ([_vp, _c_int, _c_int, _vp, _vp, _vp, _vp, _c_ll, _c_ll, _vp, _vp, _vp, _vp, _c_ll, _c_ll,
                          _vp, _vp, _c_ll, _c_ll, _vp, _c_int, _c_d, _vp, _vp, _c_ll, _c_ll, _vp, _vp, _vp], _c_int),
    "hbem_refine_async": ([_c_int, _c_int, _vp, _vp, _c_ll, _c_ll, _vp, _vp, _c_ll, _vp, _c_ll, _vp, _vp, _c_ll, _vp,
                           _vp, _c_ll, _c_d, _c_int, _vp, _vp, _vp], _c_int),
    "hbem_field": ([_vp, _c_int, _vp, _vp, _vp, _c_ll, _vp, _vp, _c_ll, _vp, _c_int, _vp, _vp, _c_ll, _vp], _c_int),
    "hbem_reduce_tag_avg": ([_vp, _c_int, _vp, _vp, _c_ll, _vp, _c_int, _vp, _vp], _c_int),
    "hbem_solve_batch": ([_vp, _c_int, _vp, _vp, _vp, _vp, _vp, _c_int, _vp, _c_int, _c_int, _c_d, _c_int, _vp, _vp,
                          _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp], _c_int),
    "hbem_session_set_aperture": ([_vp, _c_int], _c_int),
    "hbem_set_tuning": ([_c_int, _c_int], _c_int),
    "hbem_matrix_norm1": ([_c_int, _c_int, _vp, _vp, _c_ll, _c_ll, _vp, _vp], _c_int),
    "hbem_lu_rcond": ([_c_int, _c_int, _vp, _vp, _c_ll, _c_ll, _vp, _vp, _vp], _c_int),
    "hbem_get_tuning": ([_c_int], _c_int),
    "hbem_reduce_tag_avg_device": ([_vp, _c_int, _vp, _vp, _c_ll, _vp, _c_int, _vp, _vp], _c_int),
    "hbem_session_set_vertices": ([_vp, _vp, _vp, _vp], _c_int),
    "hbem_field_adjoint": ([_vp, _c_int, _vp, _vp, _c_int, _vp, _vp, _c_ll, _vp, _vp, _c_ll, _vp], _c_int),
    "hbem_field_backward": ([_vp, _c_int, _vp, _vp, _c_int, _vp, _vp, _c_ll, _vp, _vp, _c_ll, _vp, _vp, _c_ll, _vp,
                             _vp], _c_int),
    "hbem_assemble_backward": ([_vp, _c_int, _vp, _vp, _vp, _vp, _c_ll, _vp, _vp, _c_ll, _vp, _vp, _c_ll, _vp, _vp],
                               _c_int),
    "hbem_coupled_ib_augment": ([_vp, _c_int, _vp, _vp, _vp, _vp, _vp, _vp, _c_ll, _c_ll, _vp, _vp], _c_int),
    "hbem_aperture_assemble": ([_vp, _c_int, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp], _c_int),
    "hbem_coupled_ib_schur": ([_vp, _c_int, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp], _c_int),
    "hbem_coupled_ib_field": ([_vp, _c_int, _vp, _vp, _vp, _vp, _vp, _vp, _c_int, _vp, _vp, _vp, _vp, _vp], _c_int),
    "hbem_assemble_f64": ([_vp, _c_int, _vp, _vp, _vp, _vp, _c_ll, _vp, _vp, _vp, _vp, _c_ll, _c_ll, _vp, _vp, _c_ll,
                           _c_int, _vp], _c_int),
    "hbem_field_f64": ([_vp, _c_int, _vp, _vp, _vp, _c_ll, _vp, _vp, _c_ll, _vp, _c_int, _vp, _vp, _c_ll, _vp],
                       _c_int),
    "hbem_solve_status": ([_vp], _c_int),
    "hbem_session_set_near_quadrature": ([_vp, _c_int, _c_d], _c_int),
    "hbem_aperture_assemble_f64": ([_vp, _c_int, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp], _c_int),
    "hbem_coupled_ib_field_f64": ([_vp, _c_int, _vp, _vp, _vp, _vp, _c_int, _vp, _vp, _vp], _c_int),
    "hbem_assemble_multi": ([_vp, _c_int, _vp, _vp, _c_int, _vp, _vp, _c_ll, _c_ll, _vp, _vp, _vp, _vp, _c_ll, _c_ll,
                             _vp, _vp, _c_ll, _c_ll, _c_int, _vp], _c_int),
    "hbem_solve_batch_multi": ([_vp, _c_int, _c_int, _vp, _vp, _vp, _vp, _vp, _c_int, _vp, _c_int, _c_int, _c_d,
                                _c_int, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp], _c_int),
    "hbem_lu_factor_f64": ([_c_int, _c_int, _vp, _vp, _c_ll, _c_ll, _vp, _c_ll, _vp, _vp], _c_int),
    "hbem_lu_solve_f64": ([_c_int, _c_int, _c_int, _vp, _vp, _c_ll, _c_ll, _vp, _c_ll, _vp, _vp, _c_ll, _c_ll,
                           _c_int, _vp], _c_int),
}

_LIB: ctypes.CDLL | None = None


def load_library(path: str | os.PathLike | None = None) -> ctypes.CDLL:
    """Load ``libhbem.so`` (built in-tree) and declare every exported signature."""
    global _LIB
    if _LIB is not None and path is None:
        return _LIB
    p = Path(path) if path is not None else LIB_PATH
    if not p.exists():
        raise BackendUnavailable(
            f"{p} is not built; run `python -m hornlab_metal_bem_b200.csrc.build` (nvcc, sm_100a)"
        )
    lib = ctypes.CDLL(str(p))
    for name, (args, res) in _SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    if path is None:
        _LIB = lib
    return lib


def last_error(lib: ctypes.CDLL | None = None) -> str:
    lib = lib or load_library()
    buf = ctypes.create_string_buffer(2048)
    lib.hbem_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def _case_flags(k_re: float, k_im: float, *, robin: bool = False, coupled: bool = False,
                field_k: float | None = None) -> dict:
    """Per-case capability keys of the reference helper's case results, present only when they apply
    (``main.swift:9749-9761``): ``complex_k`` with ``assembly_k_imag_f32`` for a complex wavenumber,
    ``robin_boundary`` (and ``field_uses_total_neumann`` without the coupled baffle) for Robin faces,
    ``field_k_real_f32`` when the field wavenumber differs from the assembly one."""
    out: dict = {}
    if k_im != 0.0:
        out["assembly_k_imag_f32"] = float(k_im)
        out["complex_k"] = True
    if robin:
        out["robin_boundary"] = True
        if not coupled:
            out["field_uses_total_neumann"] = True
    if field_k is not None and float(field_k) != float(k_re):
        out["field_k_real_f32"] = float(field_k)
    return out


def solve_mode(precision: str, dense_solve_dtype: str = "float32") -> str:
    """The dense-solve variant of a case: ``"fp64"`` for ``dense_solve_dtype="float64"`` (complex128 LU of the
    widened FP32 system, the reference's zgesv path), else ``"mixed"`` (BF16x3 tensor-core LU) or ``"plain"``
    (FP32 LU, the reference's cgesv); plain and mixed are followed by FP64-residual refinement when
    ``refine_max_iterations`` > 0."""
    if dense_solve_dtype == "float64":
        return "fp64"
    return "mixed" if precision == "mixed" else "plain"


SOLVE_IMPL = {"plain": "hbem_blocked_lu_fp32", "mixed": "hbem_blocked_lu_bf16x3", "fp64": "hbem_blocked_lu_fp64"}


def matrix_ld(n: int) -> int:
    """Leading dimension of the dense FP32 matrices: ``n`` rounded up to 4 floats, so rows start on 16-byte
    boundaries and the LU's trailing updates move C as float4 (as ``hbem_solve_batch`` lays them out)."""
    return (int(n) + 3) & ~3


def solve_impl(mode: str, refined: bool) -> str:
    """Diagnostics name of the dense solve: a refined plain solve factors with the TF32x3 tensor-core bulk update."""
    if not refined:
        return SOLVE_IMPL[mode]
    return (SOLVE_IMPL[mode] + "_tf32x3" if mode == "plain" else SOLVE_IMPL[mode]) + "_refined"


NEAR_QUADRATURE_ENV = "HORNLAB_METAL_BEM_NATIVE_NEAR_QUADRATURE"


def parse_near_quadrature(raw) -> tuple[int, float] | None:
    """The reference's near-quadrature setting (``main.swift:5024-5054``): unset, "" or "0" = off; "1" / "2" =
    that subdivision level at threshold 1.5; "<level>:<threshold>" with level 1 or 2 and a finite positive
    threshold.  A (level, threshold) tuple passes through."""
    if raw is None:
        return None
    if isinstance(raw, tuple):
        level, threshold = int(raw[0]), float(raw[1])
        if level == 0:
            return None
        if level in (1, 2) and math.isfinite(threshold) and threshold > 0.0:
            return level, threshold
    else:
        text = str(raw).strip()
        if text in ("", "0"):
            return None
        if text in ("1", "2"):
            return int(text), 1.5
        parts = text.split(":")
        if len(parts) == 2 and parts[0] in ("1", "2"):
            try:
                threshold = float(parts[1])
            except ValueError:
                threshold = float("nan")
            if math.isfinite(threshold) and threshold > 0.0:
                return int(parts[0]), threshold
    raise ValueError(f"{NEAR_QUADRATURE_ENV} must be unset, '0', '1', '2', or '<level>:<positive threshold>' "
                     "with level 1...2")


def _refines(mode: str, max_iter) -> bool:
    return mode == "mixed" or (mode == "plain" and int(max_iter) > 0)


def check(status: int, what: str, lib: ctypes.CDLL | None = None) -> int:
    if status < 0:
        raise RuntimeError(f"{what} failed ({status}): {last_error(lib)}")
    return status


def _np_ptr(a: np.ndarray | None):
    return None if a is None else ctypes.c_void_p(a.ctypes.data)


def _t_ptr(t):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def _stream_ptr(stream=None):
    import torch

    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


def require_cuda():
    import torch

    if not torch.cuda.is_available():
        raise BackendUnavailable("no CUDA device is visible; the B200 path has no CPU fallback")
    return torch


@dataclass
class CaseResult:
    """One solved frequency (the reference's ``DenseSolveFieldResult``, in memory)."""

    frequency_hz: float
    field: np.ndarray                      # (N_obs,) complex64
    impedance: complex | None
    surface_pressure_avg: dict[int, complex] | None
    surface_pressure: np.ndarray | None    # (n_dof,) complex64
    assembly_s: float
    dense_solve_s: float
    field_s: float
    lapack_info: int
    diagnostics: dict[str, Any] = field(default_factory=dict)
    extra_sources: tuple = ()              # ExtraSourceResult per extra velocity source


@dataclass
class ExtraSourceResult:
    """Outputs of one extra velocity source sharing a case's assembled and factored matrix (the reference's
    ``ExtraSourceSolveResult``, ``hornlab_metal_bem/metal/session.py:330-350``, in memory)."""

    source_index: int                      # 1-based: the primary source is 0
    field: np.ndarray                      # (N_obs,) complex64
    impedance: complex | None
    surface_pressure_avg: dict[int, complex] | None
    surface_pressure: np.ndarray | None
    refine_iterations: int = 0
    refine_residual_rel: float | None = None
    chief_residual_rel: float | None = None   # CHIEF solves: ||s (C p - d)|| / ||b|| of this source


MAX_SOURCES_PER_PASS = 8


class NativeSession:
    """One mesh resident on one GPU (``hbem_session``)."""

    def __init__(self, geometry_buffers: GeometryBuffers, *, symmetry_plane: str | None = None,
                 aperture_tag: int | None = None, velocity_source_tags=None, check_open_edges: bool = True,
                 device: int | None = None, near_quadrature=None):
        torch = require_cuda()
        self.lib = load_library()
        self.buffers = geometry_buffers
        self.symmetry_plane = validate_native_symmetry_plane(
            geometry_buffers, symmetry_plane, check_open_edges=check_open_edges
        )
        self.aperture_tag = validate_native_infinite_baffle_aperture(
            geometry_buffers, aperture_tag, velocity_source_tags=velocity_source_tags,
            symmetry_plane=self.symmetry_plane,
        )
        self.sym_code = SYMMETRY_CODES[self.symmetry_plane]
        self.device = torch.cuda.current_device() if device is None else int(device)
        b = geometry_buffers
        self._host = [
            np.ascontiguousarray(b.vertices_3xn_f32, dtype=np.float32),
            np.ascontiguousarray(b.triangles_3xm_i32, dtype=np.int32),
            np.ascontiguousarray(b.p1_local2global_i32, dtype=np.int32),
            np.ascontiguousarray(b.physical_tags_i32, dtype=np.int32),
            np.ascontiguousarray(b.triangle_areas_f32, dtype=np.float32),
            np.ascontiguousarray(b.triangle_normals_3xm_f32, dtype=np.float32),
        ]
        v, t, l2g, tags, areas, normals = self._host
        handle = ctypes.c_void_p()
        t0 = time.perf_counter()
        check(self.lib.hbem_session_create(
            _np_ptr(v), v.shape[1], _np_ptr(t), t.shape[1], _np_ptr(l2g), int(b.p1_dof_count), _np_ptr(tags),
            _np_ptr(areas), _np_ptr(normals), self.sym_code, self.device, ctypes.byref(handle)),
            "hbem_session_create", self.lib)
        self.setup_s = time.perf_counter() - t0
        self.handle = handle
        self.n_dof = int(b.p1_dof_count)
        self.n_triangles = int(t.shape[1])
        self.m_aperture = 0
        if self.aperture_tag is not None:
            check(self.lib.hbem_session_set_aperture(self.handle, int(self.aperture_tag)),
                  "hbem_session_set_aperture", self.lib)
            self.m_aperture = self.query("aperture_triangles")
        # near-field subdivision: argument, else the reference's environment variable
        self.near_quadrature = None
        near = parse_near_quadrature(near_quadrature if near_quadrature is not None
                                     else os.environ.get(NEAR_QUADRATURE_ENV))
        if near is not None:
            t1 = time.perf_counter()
            check(self.lib.hbem_session_set_near_quadrature(self.handle, near[0], near[1]),
                  "hbem_session_set_near_quadrature", self.lib)
            self.near_quadrature = {"level": near[0], "threshold": near[1],
                                    "pair_count": self.query("near_pairs"), "seconds": time.perf_counter() - t1}

    # -- lifecycle -------------------------------------------------------------
    @classmethod
    def create_session(cls, *, geometry_buffers, symmetry_plane=None, aperture_tag=None, velocity_source_tags=None,
                       check_open_edges=True, device=None, near_quadrature=None, **_ignored) -> "NativeSession":
        return cls(geometry_buffers, symmetry_plane=symmetry_plane, aperture_tag=aperture_tag,
                   velocity_source_tags=velocity_source_tags, check_open_edges=check_open_edges, device=device,
                   near_quadrature=near_quadrature)

    def close(self) -> None:
        if getattr(self, "handle", None) is not None and self.handle.value:
            self.lib.hbem_session_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):  # pragma: no cover - interpreter shutdown ordering
        try:
            self.close()
        except Exception:
            pass

    def query(self, key: str) -> int:
        out = ctypes.c_longlong()
        check(self.lib.hbem_session_query(self.handle, QUERY_KEYS[key], ctypes.byref(out)), "hbem_session_query")
        return int(out.value)

    def pair_plan(self) -> dict[str, int]:
        c, e, v = self.query("coincident"), self.query("edge"), self.query("vertex")
        return {"coincident": c, "edge": e, "vertex": v, "total": c + e + v}

    # -- device primitives (torch tensors in, torch tensors out) ---------------
    def assemble(self, k_re, q, *, k_imag=None, beta=None, flags: int = HBEM_ASM_CORRECTED, stream=None):
        """Return ``(A_re, A_im, b_re, b_im)`` float32 CUDA tensors of shape (F, n, n) / (F, n)."""
        torch = require_cuda()
        k_re = np.ascontiguousarray(np.atleast_1d(k_re), dtype=np.float32)
        F = k_re.shape[0]
        k_im = None if k_imag is None else np.ascontiguousarray(np.atleast_1d(k_imag), dtype=np.float32)
        dev = torch.device("cuda", self.device)
        qr, qi = self._split_device(q, (F, self.n_triangles), dev)
        br_, bi_ = (None, None) if beta is None else self._split_device(beta, (self.n_triangles,), dev)
        n = self.n_dof
        Ar = torch.empty((F, n, n), dtype=torch.float32, device=dev)
        Ai = torch.empty_like(Ar)
        b_re = torch.empty((F, n), dtype=torch.float32, device=dev)
        b_im = torch.empty_like(b_re)
        check(self.lib.hbem_assemble(
            self.handle, F, _np_ptr(k_re), _np_ptr(k_im), _t_ptr(qr), _t_ptr(qi), self.n_triangles, _t_ptr(br_),
            _t_ptr(bi_), _t_ptr(Ar), _t_ptr(Ai), n, n * n, _t_ptr(b_re), _t_ptr(b_im), n, flags | HBEM_ASM_ZERO,
            _stream_ptr(stream)), "hbem_assemble", self.lib)
        return Ar, Ai, b_re, b_im

    def assemble_f64(self, k_re, q, *, k_imag=None, beta=None, flags: int = HBEM_ASM_CORRECTED, stream=None):
        """The FP64 twin of :meth:`assemble` (``hbem_assemble_f64``): float64 CUDA tensors
        ``(A_re, A_im, b_re, b_im)`` of shape (F, n, n) / (F, n), the same discretisation in double precision."""
        torch = require_cuda()
        k_re = np.ascontiguousarray(np.atleast_1d(k_re), dtype=np.float64)
        F = k_re.shape[0]
        k_im = None if k_imag is None else np.ascontiguousarray(np.atleast_1d(k_imag), dtype=np.float64)
        dev = torch.device("cuda", self.device)
        qz = np.asarray(q).reshape(F, self.n_triangles)
        qr = torch.tensor(np.ascontiguousarray(qz.real, dtype=np.float64), device=dev)
        qi = torch.tensor(np.ascontiguousarray(qz.imag, dtype=np.float64), device=dev)
        br_ = bi_ = None
        if beta is not None:
            bz = np.asarray(beta).reshape(self.n_triangles)
            br_ = torch.tensor(np.ascontiguousarray(bz.real, dtype=np.float64), device=dev)
            bi_ = torch.tensor(np.ascontiguousarray(bz.imag, dtype=np.float64), device=dev)
        n = self.n_dof
        Ar = torch.empty((F, n, n), dtype=torch.float64, device=dev)
        Ai = torch.empty_like(Ar)
        b_re = torch.empty((F, n), dtype=torch.float64, device=dev)
        b_im = torch.empty_like(b_re)
        check(self.lib.hbem_assemble_f64(
            self.handle, F, _np_ptr(k_re), _np_ptr(k_im), _t_ptr(qr), _t_ptr(qi), self.n_triangles, _t_ptr(br_),
            _t_ptr(bi_), _t_ptr(Ar), _t_ptr(Ai), n, n * n, _t_ptr(b_re), _t_ptr(b_im), n, flags | HBEM_ASM_ZERO,
            _stream_ptr(stream)), "hbem_assemble_f64", self.lib)
        return Ar, Ai, b_re, b_im

    def field_f64(self, k_re, p, q, obs_3xn, stream=None):
        """The FP64 twin of :meth:`field`: p (F, n) and q (F, T) complex arrays or tensors in, (F, N) complex128
        CUDA tensor out."""
        torch = require_cuda()
        k_re = np.ascontiguousarray(np.atleast_1d(k_re), dtype=np.float64)
        F = k_re.shape[0]
        dev = torch.device("cuda", self.device)

        def planes(z, shape):
            z = torch.as_tensor(z, device=dev).reshape(shape)
            if z.is_complex():
                return z.real.double().contiguous(), z.imag.double().contiguous()
            return z.double().contiguous(), torch.zeros(shape, dtype=torch.float64, device=dev)

        pr, pi = planes(p, (F, self.n_dof))
        qr, qi = planes(q, (F, self.n_triangles))
        obs = torch.as_tensor(np.ascontiguousarray(obs_3xn, dtype=np.float32), device=dev).contiguous()
        N = obs.shape[1]
        out_re = torch.empty((F, N), dtype=torch.float64, device=dev)
        out_im = torch.empty_like(out_re)
        check(self.lib.hbem_field_f64(
            self.handle, F, _np_ptr(k_re), _t_ptr(pr), _t_ptr(pi), self.n_dof, _t_ptr(qr), _t_ptr(qi),
            self.n_triangles, _t_ptr(obs), N, _t_ptr(out_re), _t_ptr(out_im), N, _stream_ptr(stream)),
            "hbem_field_f64", self.lib)
        return torch.complex(out_re, out_im)

    def reference_solve_f64(self, k_re, q, obs_3xn, *, k_imag=None, beta=None):
        """The FP64 path of one batch: corrected assembly, complex128 LU and solve, field, all in double
        precision on the GPU.  Returns (surface pressure (F, n), field (F, N)) as complex128 CUDA tensors; the
        error every FP32 result states is measured against these."""
        Ar, Ai, br, bi = self.assemble_f64(k_re, q, k_imag=k_imag, beta=beta)
        F = Ar.shape[0]
        x_re, x_im = lu_solve_f64(Ar, Ai, br, bi)
        p = torch_complex(x_re, x_im)
        qz = np.asarray(q).reshape(F, self.n_triangles).astype(np.complex128)
        if beta is not None:
            # the field's Neumann data on Robin faces: q + i k beta p_avg (main.swift:1646-1674)
            l2g = np.asarray(self.buffers.p1_local2global_i32)
            k = np.atleast_1d(k_re).astype(np.float64)[:, None]
            ki = (np.zeros_like(k) if k_imag is None else np.atleast_1d(k_imag).astype(np.float64)[:, None])
            p_h = p.cpu().numpy()
            qz = qz + (1j * k - ki) * np.asarray(beta).reshape(1, -1) * p_h[:, l2g].mean(axis=2)
        return p, self.field_f64(k_re, p, qz, obs_3xn)

    def coupled_reference_solve_f64(self, k_re, q, obs_3xn, *, k_imag=None, field_k=None):
        """The coupled infinite baffle on the FP64 path, one frequency at a time: FP64 corrected assembly of A
        and b, FP64 aperture projections S_ia (at k) and S_aa (at the real field wavenumber), the augmented
        system [[A, -S_ia], [P_avg, -2 S_aa]] [p; q_a] = [b; 0] (``main.swift:7504-7595``) factored by the
        complex128 LU, and the FP64 Rayleigh field of q_a.  Returns complex128 numpy arrays p (F, n),
        q_a (F, m) and field (F, N)."""
        torch = require_cuda()
        if self.m_aperture <= 0:
            raise ValueError("session has no aperture_tag")
        k_re = np.atleast_1d(np.asarray(k_re, dtype=np.float64))
        F = k_re.shape[0]
        k_im = None if k_imag is None else np.atleast_1d(np.asarray(k_imag, dtype=np.float64))
        kf = k_re if field_k is None else np.atleast_1d(np.asarray(field_k, dtype=np.float64))
        n, m = self.n_dof, self.m_aperture
        N = n + m
        dev = torch.device("cuda", self.device)
        q = np.asarray(q).reshape(F, self.n_triangles)
        obs = torch.as_tensor(np.ascontiguousarray(obs_3xn, dtype=np.float32), device=dev).contiguous()
        n_obs = int(obs.shape[1])
        l2g = torch.as_tensor(np.asarray(self.buffers.p1_local2global_i32, dtype=np.int64), device=dev)
        ap = np.flatnonzero(np.asarray(self.buffers.physical_tags_i32) == int(self.aperture_tag))
        rows_p = torch.arange(m, device=dev).repeat_interleave(3)
        cols_p = l2g[torch.as_tensor(ap, device=dev)].reshape(-1)
        out_p, out_qa, out_f = [], [], []
        for f in range(F):
            kr1 = np.ascontiguousarray(k_re[f:f + 1])
            ki1 = None if k_im is None else np.ascontiguousarray(k_im[f:f + 1])
            kf1 = np.ascontiguousarray(kf[f:f + 1])
            Ar, Ai, br, bi = self.assemble_f64(kr1, q[f:f + 1], k_imag=ki1)
            sia_r = torch.empty((1, n, m), dtype=torch.float64, device=dev)
            sia_i, saa_r, saa_i = torch.empty_like(sia_r), torch.empty((1, m, m), dtype=torch.float64,
                                                                       device=dev), None
            saa_i = torch.empty_like(saa_r)
            check(self.lib.hbem_aperture_assemble_f64(self.handle, 1, _np_ptr(kr1), _np_ptr(ki1), _np_ptr(kf1),
                                                      _t_ptr(sia_r), _t_ptr(sia_i), _t_ptr(saa_r), _t_ptr(saa_i),
                                                      _stream_ptr()), "hbem_aperture_assemble_f64", self.lib)
            Kr = torch.zeros((1, N, N), dtype=torch.float64, device=dev)
            Ki = torch.zeros_like(Kr)
            Kr[0, :n, :n], Ki[0, :n, :n] = Ar[0], Ai[0]
            del Ar, Ai
            Kr[0, :n, n:], Ki[0, :n, n:] = -sia_r[0], -sia_i[0]
            Kr[0].index_put_((n + rows_p, cols_p), torch.full_like(rows_p, 1.0 / 3.0, dtype=torch.float64),
                             accumulate=True)
            Kr[0, n:, n:], Ki[0, n:, n:] = -2.0 * saa_r[0], -2.0 * saa_i[0]
            rr = torch.zeros((1, N), dtype=torch.float64, device=dev)
            ri = torch.zeros_like(rr)
            rr[0, :n], ri[0, :n] = br[0], bi[0]
            xr, xi = lu_solve_f64(Kr, Ki, rr, ri)
            del Kr, Ki
            qa_r, qa_i = xr[:, n:].contiguous(), xi[:, n:].contiguous()
            fr = torch.empty((1, n_obs), dtype=torch.float64, device=dev)
            fi = torch.empty_like(fr)
            check(self.lib.hbem_coupled_ib_field_f64(self.handle, 1, _np_ptr(kf1), _t_ptr(qa_r), _t_ptr(qa_i),
                                                     _t_ptr(obs), n_obs, _t_ptr(fr), _t_ptr(fi), _stream_ptr()),
                  "hbem_coupled_ib_field_f64", self.lib)
            out_p.append(torch.complex(xr[0, :n], xi[0, :n]).cpu().numpy())
            out_qa.append(torch.complex(qa_r[0], qa_i[0]).cpu().numpy())
            out_f.append(torch.complex(fr[0], fi[0]).cpu().numpy())
        return np.array(out_p), np.array(out_qa), np.array(out_f)

    @staticmethod
    def _split_device(z, shape, dev):
        import torch

        if isinstance(z, tuple):
            return z
        arr = np.asarray(z).reshape(shape)
        re = torch.tensor(np.ascontiguousarray(arr.real, dtype=np.float32), device=dev).contiguous()
        im = torch.tensor(np.ascontiguousarray(arr.imag, dtype=np.float32), device=dev).contiguous()
        return re, im

    def field(self, k_re, p_re, p_im, q, obs_3xn, stream=None):
        torch = require_cuda()
        k_re = np.ascontiguousarray(np.atleast_1d(k_re), dtype=np.float32)
        F = k_re.shape[0]
        dev = p_re.device
        qr, qi = self._split_device(q, (F, self.n_triangles), dev)
        p_re, p_im = p_re.reshape(F, self.n_dof).contiguous(), p_im.reshape(F, self.n_dof).contiguous()
        obs = torch.as_tensor(np.ascontiguousarray(obs_3xn, dtype=np.float32), device=dev).contiguous()
        N = obs.shape[1]
        out_re = torch.empty((F, N), dtype=torch.float32, device=dev)
        out_im = torch.empty_like(out_re)
        check(self.lib.hbem_field(
            self.handle, F, _np_ptr(k_re), _t_ptr(p_re), _t_ptr(p_im), self.n_dof, _t_ptr(qr), _t_ptr(qi),
            self.n_triangles, _t_ptr(obs), N, _t_ptr(out_re), _t_ptr(out_im), N, _stream_ptr(stream)), "hbem_field",
            self.lib)
        return out_re, out_im

    def tag_average(self, p_re, p_im, tags, stream=None):
        torch = require_cuda()
        tags = np.ascontiguousarray(tags, dtype=np.int32)
        F = p_re.shape[0]
        p_re, p_im = p_re.reshape(F, self.n_dof).contiguous(), p_im.reshape(F, self.n_dof).contiguous()
        out = torch.empty((F, tags.shape[0], 2), dtype=torch.float64, device=p_re.device)
        check(self.lib.hbem_reduce_tag_avg(
            self.handle, F, _t_ptr(p_re), _t_ptr(p_im), self.n_dof, _np_ptr(tags), tags.shape[0], _t_ptr(out),
            _stream_ptr(stream)), "hbem_reduce_tag_avg", self.lib)
        return out

    # -- the reference-facing batched operation -------------------------------
    def assemble_solve_evaluate_standard_neumann_batch(
        self,
        frequency_hz,
        k_real_f32,
        neumann_dp0,
        observation_points,
        *,
        k_imag_f32=None,
        source_tags=None,
        impedance_source_tag=None,
        write_surface_pressure: bool = False,
        dense_solve_dtype: str = "float32",
        precision: str = "plain",
        refine_tolerance: float = 1e-6,
        refine_max_iterations: int = 10,
        timings_out: dict | None = None,
        compute_rcond: bool = True,
        impedance_sources=None,
        extra_neumann_dp0=None,
        extra_impedance_source_tags=None,
        chief_points=None,
        chief_weight: float = 1.0,
        **_ignored,
    ) -> list[CaseResult]:
        """Assemble, factor, solve and evaluate every frequency in one native call.

        Same argument meaning as the reference (``native.py:737-764``):
        ``frequency_hz`` (F,), ``k_real_f32`` (F,) float32 wavenumbers,
        ``neumann_dp0`` (F, T) complex DP0 Neumann data, ``observation_points``
        (3, N) or (N, 3).  ``dense_solve_dtype="float64"`` factors the widened
        system in complex128 (the reference's zgesv path).  Otherwise the FP32
        (``precision="plain"``) or BF16x3 (``"mixed"``) LU solution is refined
        with FP64 residuals (``refine_tolerance``, at most
        ``refine_max_iterations`` passes, stopping when a pass no longer lowers
        the residual: the reference's HORNLAB_METAL_BEM_NATIVE_DENSE_SOLVE_REFINE
        passes, main.swift:6964-7070); ``refine_max_iterations=0`` leaves the
        plain LU solution as cgesv gives it.  ``compute_rcond`` adds the
        1-norm condition estimate of each matrix (``dense_solve_rcond``), as the
        reference computes with cgecon for every case.

        ``chief_points`` (3, m) interior points switch every case to the CHIEF least-squares solve
        (``hbem_chief_lstsq``: the boundary system stacked on the interior collocation rows, weighted by
        ``chief_weight``, solved in complex128; the reference's zgels path, ``main.swift:1897-2036,
        7186-7409``); each result's diagnostics carry ``chief_residual_rel``.

        ``extra_neumann_dp0`` (n_extra, F, T) adds velocity sources that share
        each frequency's assembled and factored matrix (the reference's
        multi-RHS batch, ``native.py:775-779``): one assembly pass evaluates
        the kernel once for the matrix and every source's right-hand side,
        one LU per frequency, one solve per source.  Their outputs are each
        result's ``extra_sources``; ``extra_impedance_source_tags`` names the
        tag whose average becomes each extra source's ``impedance``.
        """
        freqs = np.ascontiguousarray(np.atleast_1d(frequency_hz), dtype=np.float64)
        F = freqs.shape[0]
        k_re = np.ascontiguousarray(np.atleast_1d(k_real_f32), dtype=np.float32)
        if k_re.shape != (F,):
            raise ValueError("k_real_f32 must have one value per frequency")
        extra = None
        if extra_neumann_dp0 is not None:
            extra = np.asarray(extra_neumann_dp0)
            if extra.ndim != 3 or extra.shape[1:] != (F, self.n_triangles):
                raise ValueError(f"extra_neumann_dp0 must have shape (n_extra, {F}, {self.n_triangles}), "
                                 f"got {extra.shape}")
            if extra.shape[0] == 0:
                raise ValueError("extra_neumann_dp0 must be None or non-empty")
            if not np.all(np.isfinite(extra)):
                raise ValueError("extra_neumann_dp0 must contain only finite values")
            if extra_impedance_source_tags is not None and len(extra_impedance_source_tags) != extra.shape[0]:
                raise ValueError("extra_impedance_source_tags must name one tag (or None) per extra source")
        elif extra_impedance_source_tags is not None:
            raise ValueError("extra_impedance_source_tags requires extra_neumann_dp0")
        if chief_points is not None:
            pts = np.asarray(chief_points, dtype=np.float32)
            if pts.ndim != 2 or pts.shape[0] != 3:
                raise ValueError("chief_points must have shape (3, m)")
            if pts.shape[1] == 0:
                raise ValueError("chief_points must be non-empty when set")
            if not np.all(np.isfinite(pts)):
                raise ValueError("chief_points must be finite")
            if not (np.isfinite(chief_weight) and float(chief_weight) > 0):
                raise ValueError("chief_weight must be finite and positive")
            per = None
            if impedance_sources:
                per = impedance_sources if isinstance(impedance_sources, list) else [impedance_sources] * F
                if len(per) != F:
                    raise ValueError(f"impedance_sources list must have one dict per frequency ({F}), got {len(per)}")
                if not any(per):
                    per = None
            q = np.asarray(neumann_dp0)
            if q.shape != (F, self.n_triangles) or not np.all(np.isfinite(q)):
                raise ValueError(f"neumann_dp0 must be finite with shape {(F, self.n_triangles)}")
            qs = q[None] if extra is None else np.concatenate([q[None], extra], axis=0)
            return self._chief_batch(freqs, k_re, k_imag_f32, qs, observation_points, per, pts, float(chief_weight),
                                     source_tags=source_tags, impedance_source_tag=impedance_source_tag,
                                     extra_tags=(list(extra_impedance_source_tags) if extra_impedance_source_tags
                                                 else [None] * (qs.shape[0] - 1)),
                                     write_surface_pressure=write_surface_pressure, timings_out=timings_out)
        if impedance_sources:
            per = impedance_sources if isinstance(impedance_sources, list) else [impedance_sources] * F
            if len(per) != F:
                raise ValueError(f"impedance_sources list must have one dict per frequency ({F}), got {len(per)}")
            if any(per) and extra is not None:
                raise BackendUnavailable("extra_neumann_dp0 with impedance_sources (Robin) is solved one source at a "
                                         "time; call once per source")
            if any(per):
                return self._robin_batch(freqs, k_re, k_imag_f32, neumann_dp0, observation_points, per,
                                         source_tags=source_tags, impedance_source_tag=impedance_source_tag,
                                         write_surface_pressure=write_surface_pressure,
                                         precision=solve_mode(precision, dense_solve_dtype),
                                         refine_tolerance=refine_tolerance,
                                         refine_max_iterations=refine_max_iterations, timings_out=timings_out,
                                         compute_rcond=compute_rcond)
        k_im = None if k_imag_f32 is None else np.ascontiguousarray(np.atleast_1d(k_imag_f32), dtype=np.float32)
        q = np.asarray(neumann_dp0)
        if q.shape != (F, self.n_triangles):
            raise ValueError(f"neumann_dp0 must have shape {(F, self.n_triangles)}, got {q.shape}")
        if not np.all(np.isfinite(q)):
            raise ValueError("neumann_dp0 must be finite")
        obs = np.asarray(observation_points, dtype=np.float64)
        if obs.ndim != 2 or 3 not in obs.shape:
            raise ValueError("observation_points must have shape (3, N) or (N, 3)")
        if obs.shape[0] != 3:
            obs = obs.T
        obs = np.ascontiguousarray(obs, dtype=np.float32)
        N = obs.shape[1]
        tags = list(source_tags or [])
        imp_tag = impedance_source_tag
        extra_tags = list(extra_impedance_source_tags) if extra is not None and extra_impedance_source_tags else []
        want = list(tags)
        for t in [imp_tag] + extra_tags:
            if t is not None and t not in want:
                want.append(t)
        want_arr = np.ascontiguousarray(want, dtype=np.int32) if want else np.zeros(1, np.int32)
        qs = q[None] if extra is None else np.concatenate([q[None], extra], axis=0)   # (S, F, T)
        S = qs.shape[0]
        mode = solve_mode(precision, dense_solve_dtype)
        prec = {"plain": HBEM_PREC_PLAIN, "mixed": HBEM_PREC_MIXED, "fp64": HBEM_PREC_FP64}[mode]
        max_it = 0 if mode == "fp64" else int(refine_max_iterations)
        if mode == "mixed":
            max_it = max(1, max_it)
        tol = float(refine_tolerance)
        fr = np.zeros((S, F, N), np.float32)
        fi = np.zeros((S, F, N), np.float32)
        tavg = np.zeros((S, F, max(1, len(want)), 2), np.float64)
        sr = np.zeros((S, F, self.n_dof), np.float32) if (write_surface_pressure or S > 1) else None
        si = np.zeros((S, F, self.n_dof), np.float32) if sr is not None else None
        info = np.zeros(F, np.int32)
        iters = np.zeros((S, F), np.int32)
        resid = np.zeros((S, F), np.float64)
        rcond = np.zeros(F, np.float64) if compute_rcond else None
        tms = np.zeros(4, np.float32)
        t0 = time.perf_counter()
        for s0 in range(0, S, MAX_SOURCES_PER_PASS):
            sl = slice(s0, min(S, s0 + MAX_SOURCES_PER_PASS))
            ns = sl.stop - sl.start
            qr = np.ascontiguousarray(qs[sl].real, dtype=np.float32)
            qi = np.ascontiguousarray(qs[sl].imag, dtype=np.float32)
            tpart = np.zeros(4, np.float32)
            views = [np.ascontiguousarray(a[sl]) if a is not None else None for a in (fr, fi, tavg, sr, si, iters, resid)]
            check(self.lib.hbem_solve_batch_multi(
                self.handle, F, ns, _np_ptr(k_re), _np_ptr(k_im), _np_ptr(qr), _np_ptr(qi), _np_ptr(obs), N,
                _np_ptr(want_arr), len(want), prec, tol, max_it, _np_ptr(views[0]), _np_ptr(views[1]),
                _np_ptr(views[2]), _np_ptr(views[3]), _np_ptr(views[4]), _np_ptr(info), _np_ptr(views[5]),
                _np_ptr(views[6]), _np_ptr(rcond), _np_ptr(tpart), None), "hbem_solve_batch", self.lib)
            for a, v in zip((fr, fi, tavg, sr, si, iters, resid), views):
                if a is not None:
                    a[sl] = v
            tms += tpart
        wall = time.perf_counter() - t0
        if timings_out is not None:
            timings_out.update(assembly_ms=float(tms[0]), solve_ms=float(tms[1]), field_ms=float(tms[2]),
                               total_ms=float(tms[3]), wall_s=wall, sources=S)
        per = 1.0 / F
        results = []
        for f in range(F):
            avgs = [{int(t): complex(tavg[s_, f, j, 0], tavg[s_, f, j, 1]) for j, t in enumerate(want)}
                    for s_ in range(S)]
            diag = {
                "dense_solve_impl": solve_impl(mode, max_it > 0),
                "dense_solve_dtype": dense_solve_dtype,
                "precision": precision,
                "refine_iterations": int(iters[0, f]),
                "refine_residual_rel": float(resid[0, f]) if max_it > 0 else None,
                "dense_solve_rcond": float(rcond[f]) if rcond is not None and info[f] == 0 else None,
                "assembly_mode": "corrected",
                "duffy_pairs": None,
                **_case_flags(float(k_re[f]), 0.0 if k_im is None else float(k_im[f])),
            }
            if S > 1:
                diag["multi_source"] = True
                diag["sources_sharing_factorisation"] = S
            if self.near_quadrature is not None:
                diag["near_quadrature"] = dict(self.near_quadrature)
            extras = tuple(
                ExtraSourceResult(
                    source_index=s_,
                    field=(fr[s_, f] + 1j * fi[s_, f]).astype(np.complex64),
                    impedance=(avgs[s_].get(int(extra_tags[s_ - 1]))
                               if extra_tags and extra_tags[s_ - 1] is not None else None),
                    surface_pressure_avg={int(t): avgs[s_][int(t)] for t in tags} if tags else None,
                    surface_pressure=(sr[s_, f] + 1j * si[s_, f]).astype(np.complex64) if sr is not None else None,
                    refine_iterations=int(iters[s_, f]),
                    refine_residual_rel=float(resid[s_, f]) if max_it > 0 else None,
                ) for s_ in range(1, S))
            results.append(CaseResult(
                frequency_hz=float(freqs[f]),
                field=(fr[0, f] + 1j * fi[0, f]).astype(np.complex64),
                impedance=avgs[0].get(int(imp_tag)) if imp_tag is not None else None,
                surface_pressure_avg={int(t): avgs[0][int(t)] for t in tags} if tags else None,
                surface_pressure=(None if not write_surface_pressure
                                  else (sr[0, f] + 1j * si[0, f]).astype(np.complex64)),
                assembly_s=float(tms[0]) * 1e-3 * per,
                dense_solve_s=float(tms[1]) * 1e-3 * per,
                field_s=float(tms[2]) * 1e-3 * per,
                lapack_info=int(info[f]),
                diagnostics=diag,
                extra_sources=extras,
            ))
        return results


    # -- CHIEF least squares ----------------------------------------------------
    def _chief_batch(self, freqs, k_re, k_imag_f32, qs, observation_points, per_freq, chief_pts, chief_weight, *,
                     source_tags, impedance_source_tag, extra_tags, write_surface_pressure, timings_out):
        """CHIEF sweep: the FP32 corrected assembly of every source's right-hand side (with Robin admittances
        when ``per_freq`` gives them, frequencies with equal sets sharing one launch), then
        ``hbem_chief_lstsq`` (interior collocation rows, complex128 Householder least squares of the stacked
        system), and the field and tag averages of its solution; the field's Neumann data carry the Robin
        term q + i k beta p_avg (``main.swift:1646-1674``)."""
        torch = require_cuda()
        dev = torch.device("cuda", self.device)
        st = _stream_ptr()
        F, n, T = freqs.shape[0], self.n_dof, self.n_triangles
        S = qs.shape[0]
        if S > MAX_SOURCES_PER_PASS:
            raise ValueError(f"CHIEF solves take at most {MAX_SOURCES_PER_PASS} sources per call")
        k_im = (np.zeros(F, np.float32) if k_imag_f32 is None
                else np.ascontiguousarray(np.atleast_1d(k_imag_f32), dtype=np.float32))
        obs = np.asarray(observation_points, dtype=np.float64)
        if obs.shape[0] != 3:
            obs = obs.T
        obs_t = torch.tensor(np.ascontiguousarray(obs, dtype=np.float32), device=dev)
        N = obs_t.shape[1]
        pts = np.ascontiguousarray(chief_pts, dtype=np.float32)
        m = pts.shape[1]
        tags_tri = np.asarray(self.buffers.physical_tags_i32)
        l2g = torch.as_tensor(np.asarray(self.buffers.p1_local2global_i32, dtype=np.int64), device=dev)
        tags = list(source_tags or [])
        want = list(tags)
        for t in [impedance_source_tag] + list(extra_tags):
            if t is not None and t not in want:
                want.append(t)
        out_field = np.zeros((S, F, N), np.complex64)
        out_p = np.zeros((S, F, n), np.complex64)
        out_tavg = np.zeros((S, F, max(1, len(want))), np.complex128)
        out_res = np.zeros((S, F))
        out_scale = np.zeros(F)
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
        t_asm = t_solve = t_field = 0.0
        groups, start = [], 0
        for f in range(1, F + 1):
            if f == F or (per_freq is not None and per_freq[f] != per_freq[start]):
                groups.append((start, f))
                start = f
        for g0, g1 in groups:
            Fg = g1 - g0
            sl = slice(g0, g1)
            b_re = b_im = None
            if per_freq is not None and per_freq[g0]:
                beta = np.zeros(T, np.complex64)
                for tag, bv in per_freq[g0].items():
                    beta[tags_tri == int(tag)] = complex(bv)
                b_re = torch.tensor(np.ascontiguousarray(beta.real), device=dev)
                b_im = torch.tensor(np.ascontiguousarray(beta.imag), device=dev)
            qg = qs[:, sl]
            qr = torch.tensor(np.ascontiguousarray(qg.real, dtype=np.float32), device=dev)
            qi = torch.tensor(np.ascontiguousarray(qg.imag, dtype=np.float32), device=dev)
            Ar = torch.empty((Fg, n, n), dtype=torch.float32, device=dev)
            Ai = torch.empty_like(Ar)
            br = torch.empty((S, Fg, n), dtype=torch.float32, device=dev)
            bi = torch.empty_like(br)
            kr_g, ki_g = np.ascontiguousarray(k_re[sl]), np.ascontiguousarray(k_im[sl])
            ev[0].record()
            check(self.lib.hbem_assemble_multi(
                self.handle, Fg, _np_ptr(kr_g), _np_ptr(ki_g), S, _t_ptr(qr), _t_ptr(qi), T, Fg * T, _t_ptr(b_re),
                _t_ptr(b_im), _t_ptr(Ar), _t_ptr(Ai), n, n * n, _t_ptr(br), _t_ptr(bi), n, Fg * n,
                HBEM_ASM_CORRECTED | HBEM_ASM_ZERO, st), "hbem_assemble_multi", self.lib)
            ev[1].record()
            xr = torch.empty((S, Fg, n), dtype=torch.float32, device=dev)
            xi = torch.empty_like(xr)
            res = torch.zeros((S, Fg), dtype=torch.float64, device=dev)
            scl = torch.zeros(Fg, dtype=torch.float64, device=dev)
            check(self.lib.hbem_chief_lstsq(
                self.handle, Fg, S, _np_ptr(kr_g), _np_ptr(ki_g), _t_ptr(qr), _t_ptr(qi), T, Fg * T, _t_ptr(b_re),
                _t_ptr(b_im), _t_ptr(Ar), _t_ptr(Ai), n, n * n, _t_ptr(br), _t_ptr(bi), n, Fg * n, _np_ptr(pts), m,
                chief_weight, _t_ptr(xr), _t_ptr(xi), n, Fg * n, _t_ptr(res), _t_ptr(scl), st),
                "hbem_chief_lstsq", self.lib)
            del Ar, Ai
            ev[2].record()
            for s_ in range(S):
                xs_r, xs_i = xr[s_].contiguous(), xi[s_].contiguous()
                qtr, qti = qr[s_].contiguous(), qi[s_].contiguous()
                if b_re is not None:
                    p_c = torch.complex(xs_r, xs_i)
                    p_avg = (p_c[:, l2g[:, 0]] + p_c[:, l2g[:, 1]] + p_c[:, l2g[:, 2]]) / 3.0
                    ik = torch.complex(torch.tensor(-ki_g, device=dev), torch.tensor(kr_g, device=dev))[:, None]
                    q_tot = torch.complex(qtr, qti) + ik * torch.complex(b_re, b_im)[None, :] * p_avg
                    qtr, qti = q_tot.real.contiguous(), q_tot.imag.contiguous()
                fr = torch.empty((Fg, N), dtype=torch.float32, device=dev)
                fi = torch.empty_like(fr)
                check(self.lib.hbem_field(self.handle, Fg, _np_ptr(kr_g), _t_ptr(xs_r), _t_ptr(xs_i), n,
                                          _t_ptr(qtr), _t_ptr(qti), T, _t_ptr(obs_t), N, _t_ptr(fr), _t_ptr(fi), N,
                                          st), "hbem_field", self.lib)
                tavg = self.tag_average(xs_r, xs_i, want).cpu().numpy() if want else None
                out_field[s_, sl] = (fr.cpu().numpy() + 1j * fi.cpu().numpy()).astype(np.complex64)
                out_p[s_, sl] = (xs_r.cpu().numpy() + 1j * xs_i.cpu().numpy()).astype(np.complex64)
                if tavg is not None:
                    out_tavg[s_, sl] = tavg[..., 0] + 1j * tavg[..., 1]
            ev[3].record()
            torch.cuda.synchronize()
            t_asm += ev[0].elapsed_time(ev[1])
            t_solve += ev[1].elapsed_time(ev[2])
            t_field += ev[2].elapsed_time(ev[3])
            out_res[:, sl] = res.cpu().numpy()
            out_scale[sl] = scl.cpu().numpy()
        if timings_out is not None:
            timings_out.update(assembly_ms=t_asm, solve_ms=t_solve, field_ms=t_field, total_ms=t_asm + t_solve + t_field,
                               sources=S)
        results = []
        for f in range(F):
            avgs = [{int(t): complex(out_tavg[s_, f, j]) for j, t in enumerate(want)} for s_ in range(S)]
            diag = {"dense_solve_impl": "householder_qr_lstsq_f64", "dense_solve_dtype": "float64",
                    "precision": "plain", "refine_iterations": 0, "refine_residual_rel": None,
                    "dense_solve_rcond": None, "assembly_mode": "corrected",
                    "chief_points": True, "chief_point_count": int(m), "chief_weight": float(chief_weight),
                    "chief_scale": float(out_scale[f]), "chief_residual_rel": float(out_res[0, f]),
                    **_case_flags(float(k_re[f]), float(k_im[f]), robin=per_freq is not None and bool(per_freq[f]))}
            if per_freq is not None and per_freq[f]:
                diag["robin_tags"] = sorted(int(t) for t in per_freq[f])
            if S > 1:
                diag["multi_source"] = True
                diag["sources_sharing_factorisation"] = S
            if self.near_quadrature is not None:
                diag["near_quadrature"] = dict(self.near_quadrature)
            extras = tuple(
                ExtraSourceResult(
                    source_index=s_, field=out_field[s_, f],
                    impedance=(avgs[s_].get(int(extra_tags[s_ - 1])) if extra_tags[s_ - 1] is not None else None),
                    surface_pressure_avg={int(t): avgs[s_][int(t)] for t in tags} if tags else None,
                    surface_pressure=out_p[s_, f] if write_surface_pressure else None,
                    refine_iterations=0, refine_residual_rel=None, chief_residual_rel=float(out_res[s_, f]),
                ) for s_ in range(1, S))
            results.append(CaseResult(
                frequency_hz=float(freqs[f]), field=out_field[0, f],
                impedance=avgs[0].get(int(impedance_source_tag)) if impedance_source_tag is not None else None,
                surface_pressure_avg={int(t): avgs[0][int(t)] for t in tags} if tags else None,
                surface_pressure=out_p[0, f] if write_surface_pressure else None,
                assembly_s=t_asm * 1e-3 / F, dense_solve_s=t_solve * 1e-3 / F, field_s=t_field * 1e-3 / F,
                lapack_info=0, diagnostics=diag, extra_sources=extras,
            ))
        return results

    # -- Robin (impedance) boundaries -----------------------------------------
    def _robin_batch(self, freqs, k_re, k_imag_f32, neumann_dp0, observation_points, per_freq, *, source_tags,
                     impedance_source_tag, write_surface_pressure, precision, refine_tolerance,
                     refine_max_iterations, timings_out, compute_rcond):
        """Sweep with Robin admittances beta per tag: the assembly adds the Robin terms
        (``main.swift:1731-1760, 3016``) and the field uses the Neumann data with the
        Robin contribution q + i k beta p_avg on Robin faces (``neumannWithRobin``,
        ``main.swift:1646-1674``).  Frequencies sharing one admittance set share one
        assembly launch."""
        torch = require_cuda()
        dev = torch.device("cuda", self.device)
        st = _stream_ptr()
        F, n, T = freqs.shape[0], self.n_dof, self.n_triangles
        k_im = (np.zeros(F, np.float32) if k_imag_f32 is None
                else np.ascontiguousarray(np.atleast_1d(k_imag_f32), dtype=np.float32))
        q = np.asarray(neumann_dp0).reshape(F, T)
        obs = np.asarray(observation_points, dtype=np.float64)
        if obs.shape[0] != 3:
            obs = obs.T
        obs_t = torch.tensor(np.ascontiguousarray(obs, dtype=np.float32), device=dev)
        N = obs_t.shape[1]
        tags_tri = np.asarray(self.buffers.physical_tags_i32)
        l2g = torch.as_tensor(np.asarray(self.buffers.p1_local2global_i32, dtype=np.int64), device=dev)
        tags = list(source_tags or [])
        want = tags + ([impedance_source_tag] if impedance_source_tag is not None and impedance_source_tag not in tags
                       else [])
        mode = precision  # "plain", "mixed" or "fp64" (solve_mode)
        out_field = np.zeros((F, N), np.complex64)
        out_p = np.zeros((F, n), np.complex64)
        out_tavg = np.zeros((F, max(1, len(want))), np.complex128)
        out_info = np.zeros(F, np.int64)
        out_iter = np.zeros(F, np.int64)
        out_res = np.zeros(F)
        out_rc = np.full(F, np.nan)
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
        t_asm = t_solve = t_field = 0.0
        # group consecutive frequencies with equal admittance sets
        groups, start = [], 0
        for f in range(1, F + 1):
            if f == F or per_freq[f] != per_freq[start]:
                groups.append((start, f))
                start = f
        for g0, g1 in groups:
            Fg = g1 - g0
            sl = slice(g0, g1)
            beta = np.zeros(T, np.complex64)
            for tag, b in per_freq[g0].items():
                beta[tags_tri == int(tag)] = complex(b)
            b_re = torch.tensor(np.ascontiguousarray(beta.real), device=dev)
            b_im = torch.tensor(np.ascontiguousarray(beta.imag), device=dev)
            qr, qi = self._split_device(q[sl], (Fg, T), dev)
            ld = matrix_ld(n)
            Ar = torch.empty((Fg, n, ld), dtype=torch.float32, device=dev)
            Ai = torch.empty_like(Ar)
            br = torch.empty((Fg, n), dtype=torch.float32, device=dev)
            bi = torch.empty_like(br)
            kr_g, ki_g = np.ascontiguousarray(k_re[sl]), np.ascontiguousarray(k_im[sl])
            ev[0].record()
            check(self.lib.hbem_assemble(self.handle, Fg, _np_ptr(kr_g), _np_ptr(ki_g), _t_ptr(qr), _t_ptr(qi), T,
                                         _t_ptr(b_re), _t_ptr(b_im), _t_ptr(Ar), _t_ptr(Ai), ld, n * ld, _t_ptr(br),
                                         _t_ptr(bi), n, HBEM_ASM_CORRECTED | HBEM_ASM_ZERO, st),
                  "hbem_assemble", self.lib)
            ev[1].record()
            xr, xi, info, iters, resid, rc = self._factor_solve_refine(Ar, Ai, br, bi, n, Fg, mode, refine_tolerance,
                                                                     refine_max_iterations, compute_rcond)
            del Ar, Ai
            ev[2].record()
            # Neumann data with the Robin term for the field
            p_c = torch.complex(xr, xi)
            p_avg = (p_c[:, l2g[:, 0]] + p_c[:, l2g[:, 1]] + p_c[:, l2g[:, 2]]) / 3.0
            ik = torch.complex(torch.tensor(-ki_g, device=dev), torch.tensor(kr_g, device=dev))[:, None]
            beta_t = torch.complex(b_re, b_im)[None, :]
            q_tot = torch.complex(qr, qi) + ik * beta_t * p_avg
            qtr, qti = q_tot.real.contiguous(), q_tot.imag.contiguous()
            fr = torch.empty((Fg, N), dtype=torch.float32, device=dev)
            fi = torch.empty_like(fr)
            check(self.lib.hbem_field(self.handle, Fg, _np_ptr(kr_g), _t_ptr(xr), _t_ptr(xi), n, _t_ptr(qtr),
                                      _t_ptr(qti), T, _t_ptr(obs_t), N, _t_ptr(fr), _t_ptr(fi), N, st),
                  "hbem_field", self.lib)
            tavg = self.tag_average(xr, xi, want).cpu().numpy() if want else None
            ev[3].record()
            torch.cuda.synchronize()
            t_asm += ev[0].elapsed_time(ev[1])
            t_solve += ev[1].elapsed_time(ev[2])
            t_field += ev[2].elapsed_time(ev[3])
            out_field[sl] = (fr.cpu().numpy() + 1j * fi.cpu().numpy()).astype(np.complex64)
            out_p[sl] = p_c.cpu().numpy().astype(np.complex64)
            if tavg is not None:
                out_tavg[sl] = tavg[..., 0] + 1j * tavg[..., 1]
            out_info[sl] = info.cpu().numpy()
            out_iter[sl] = iters.cpu().numpy()
            out_res[sl] = resid.cpu().numpy()
            if rc is not None:
                out_rc[sl] = rc.cpu().numpy()
        if timings_out is not None:
            timings_out.update(assembly_ms=t_asm, solve_ms=t_solve, field_ms=t_field, total_ms=t_asm + t_solve + t_field)
        results = []
        for f in range(F):
            avgs = {int(t): complex(out_tavg[f, j]) for j, t in enumerate(want)}
            results.append(CaseResult(
                frequency_hz=float(freqs[f]), field=out_field[f],
                impedance=avgs.get(int(impedance_source_tag)) if impedance_source_tag is not None else None,
                surface_pressure_avg={int(t): avgs[int(t)] for t in tags} if tags else None,
                surface_pressure=out_p[f] if write_surface_pressure else None,
                assembly_s=t_asm * 1e-3 / F, dense_solve_s=t_solve * 1e-3 / F, field_s=t_field * 1e-3 / F,
                lapack_info=int(out_info[f]),
                diagnostics={"dense_solve_impl": solve_impl(mode, _refines(mode, refine_max_iterations)),
                             "precision": "mixed" if mode == "mixed" else "plain",
                             "dense_solve_dtype": "float64" if mode == "fp64" else "float32",
                             "refine_iterations": int(out_iter[f]),
                             "refine_residual_rel": (float(out_res[f]) if _refines(mode, refine_max_iterations)
                                                     else None),
                             "dense_solve_rcond": (float(out_rc[f]) if compute_rcond and out_info[f] == 0 else None),
                             "robin_tags": sorted(int(t) for t in per_freq[f]),
                             "assembly_mode": "corrected",
                             **_case_flags(float(k_re[f]), float(k_im[f]), robin=True)},
            ))
        return results

    # -- coupled infinite baffle ---------------------------------------------
    def coupled_ib_batch(self, frequency_hz, k_real_f32, neumann_dp0, observation_points, *, k_imag_f32=None,
                         field_k_f32=None, source_tags=None, impedance_source_tag=None,
                         write_surface_pressure=False, precision="plain", refine_tolerance=1e-6,
                         refine_max_iterations=10, timings_out=None, coupled_method="auto",
                         max_chunk_bytes=None, compute_rcond=True, dense_solve_dtype="float32",
                         **_ignored) -> list[CaseResult]:
        """Coupled interior BIE + Rayleigh half-space solve (the reference's aperture_tag path).

        ``coupled_method="schur"``: A - S_ia (2 S_aa)^-1 P_avg is factored per
        frequency and the field is the Rayleigh integral of
        q_a = (2 S_aa)^-1 P_avg p (main.swift:1397-1444, 7597-7789).
        ``"augmented"``: the reference's augmented twin (main.swift:7504-7595),
        one (m + n) LU giving p and q_a together; cheaper once the aperture
        has more than a few hundred faces.  ``"auto"`` picks augmented for
        m >= AUGMENTED_MIN_APERTURE.  Frequencies are processed in chunks that
        fit ``max_chunk_bytes`` (default: half the free device memory).
        """
        torch = require_cuda()
        if self.m_aperture <= 0:
            raise ValueError("session has no aperture_tag")
        if _ignored.get("impedance_sources") and any(
                _ignored["impedance_sources"] if isinstance(_ignored["impedance_sources"], list)
                else [_ignored["impedance_sources"]]):
            raise BackendUnavailable("impedance_sources (Robin) are not supported with the coupled infinite baffle")
        if coupled_method not in ("auto", "schur", "augmented"):
            raise ValueError("coupled_method must be 'auto', 'schur' or 'augmented'")
        method = coupled_method
        if method == "auto":
            env = os.environ.get("HORNLAB_METAL_BEM_NATIVE_COUPLED_IB_SOLVE", "").strip().lower()
            if env in ("schur", "augmented"):
                method = env
            else:
                method = "augmented" if self.m_aperture >= AUGMENTED_MIN_APERTURE else "schur"
        dev = torch.device("cuda", self.device)
        freqs = np.ascontiguousarray(np.atleast_1d(frequency_hz), dtype=np.float64)
        F, n, m, T = freqs.shape[0], self.n_dof, self.m_aperture, self.n_triangles
        k_re = np.ascontiguousarray(np.atleast_1d(k_real_f32), dtype=np.float32)
        k_im = None if k_imag_f32 is None else np.ascontiguousarray(np.atleast_1d(k_imag_f32), dtype=np.float32)
        kf = k_re if field_k_f32 is None else np.ascontiguousarray(np.atleast_1d(field_k_f32), dtype=np.float32)
        q_all = np.asarray(neumann_dp0).reshape(F, T)
        obs = np.asarray(observation_points, dtype=np.float64)
        if obs.shape[0] != 3:
            obs = obs.T
        obs_t = torch.tensor(np.ascontiguousarray(obs, dtype=np.float32), device=dev)
        mode = solve_mode(precision, dense_solve_dtype)
        # dense copies per system: the factored matrix, plus the original for refinement or the FP64 twin
        copies = 3 if mode == "fp64" else (2 if _refines(mode, refine_max_iterations) else 1)
        N = n + m
        if method == "augmented":
            per_freq = 8 * (N * N * copies + n * m + m * m + 4 * N)
        else:
            per_freq = 8 * (n * n * copies + 2 * n * m + 2 * m * m + 4 * n)
        if max_chunk_bytes is None:
            free, _ = torch.cuda.mem_get_info(dev)
            max_chunk_bytes = free // 2
        chunk = int(max(1, min(F, max_chunk_bytes // per_freq)))
        tags = list(source_tags or [])
        want = tags + ([impedance_source_tag] if impedance_source_tag is not None and impedance_source_tag not in tags else [])
        parts = []
        times = np.zeros(3)
        for f0 in range(0, F, chunk):
            sl = slice(f0, min(F, f0 + chunk))
            run = self._coupled_chunk_augmented if method == "augmented" else self._coupled_chunk_schur
            parts.append(run(k_re[sl], None if k_im is None else k_im[sl], kf[sl], q_all[sl], obs_t, want,
                             mode, refine_tolerance, refine_max_iterations, times, compute_rcond))
        if timings_out is not None:
            timings_out.update(assembly_ms=times[0], solve_ms=times[1], field_ms=times[2], coupled_method=method,
                               frequency_chunk=chunk)
        cat = {key: np.concatenate([pt[key] for pt in parts]) for key in parts[0] if parts[0][key] is not None}
        out = []
        t_asm, t_solve, t_field = times
        for f in range(F):
            avgs = {int(t): complex(cat["tavg"][f, j, 0], cat["tavg"][f, j, 1]) for j, t in enumerate(want)} if want else {}
            out.append(CaseResult(
                frequency_hz=float(freqs[f]), field=cat["field"][f],
                impedance=avgs.get(int(impedance_source_tag)) if impedance_source_tag is not None else None,
                surface_pressure_avg={int(t): avgs[int(t)] for t in tags} if tags else None,
                surface_pressure=cat["p"][f] if write_surface_pressure else None,
                assembly_s=t_asm * 1e-3 / F, dense_solve_s=t_solve * 1e-3 / F, field_s=t_field * 1e-3 / F,
                lapack_info=int(cat["info"][f] or cat["info_ap"][f]),
                diagnostics={"coupled_ib": True, "ib_coupled_solve": method, "aperture_triangles": m,
                             "aperture_neumann": cat["qa"][f], "aperture_lapack_info": int(cat["info_ap"][f]),
                             "precision": precision, "dense_solve_dtype": dense_solve_dtype,
                             "dense_solve_impl": solve_impl(mode, _refines(mode, refine_max_iterations)),
                             "refine_iterations": int(cat["iters"][f]),
                             "refine_residual_rel": (float(cat["resid"][f]) if _refines(mode, refine_max_iterations)
                                                     else None),
                             "dense_solve_rcond": (float(cat["rcond"][f]) if "rcond" in cat and cat["info"][f] == 0
                                                   else None),
                             "assembly_mode": "corrected",
                             **_case_flags(float(k_re[f]), 0.0 if k_im is None else float(k_im[f]), coupled=True,
                                           field_k=float(kf[f]))},
            ))
        return out

    def _factor_solve_refine(self, Kr, Ki, br, bi, N, F, mode, tol, max_iter, rcond=False):
        """Factor and solve F systems of order N stored (F, N, lda): ``mode`` "plain" (FP32 LU) or "mixed"
        (BF16x3 LU), each refined with FP64 residuals when ``max_iter`` > 0 (mixed: at least one pass), or
        "fp64" (complex128 LU of the widened system, solution narrowed to FP32).  Returns x, info, iters, resid
        and the 1-norm reciprocal condition estimates (or None).  Kr/Ki are overwritten by FP32 factors."""
        import torch

        dev, st = Kr.device, _stream_ptr()
        lda = int(Kr.shape[2])
        anorm = rc = None
        if rcond:
            anorm = torch.empty(F, dtype=torch.float32, device=dev)
            rc = torch.empty(F, dtype=torch.float64, device=dev)
            check(self.lib.hbem_matrix_norm1(N, F, _t_ptr(Kr), _t_ptr(Ki), lda, N * lda, _t_ptr(anorm), st),
                  "hbem_matrix_norm1", self.lib)
        piv = torch.empty((F, N), dtype=torch.int32, device=dev)
        info = torch.empty(F, dtype=torch.int32, device=dev)
        iters = torch.zeros(F, dtype=torch.int32, device=dev)
        resid = torch.zeros(F, dtype=torch.float64, device=dev)
        if mode == "fp64":
            K64r, K64i = Kr.double().contiguous(), Ki.double().contiguous()
            x64r, x64i = br.double().contiguous(), bi.double().contiguous()
            check(self.lib.hbem_lu_factor_f64(N, F, _t_ptr(K64r), _t_ptr(K64i), lda, N * lda, _t_ptr(piv), N,
                                              _t_ptr(info), st), "hbem_lu_factor_f64", self.lib)
            check(self.lib.hbem_lu_solve_f64(N, 1, F, _t_ptr(K64r), _t_ptr(K64i), lda, N * lda, _t_ptr(piv), N,
                                             _t_ptr(x64r), _t_ptr(x64i), 1, N, HBEM_TRANS_N, st),
                  "hbem_lu_solve_f64", self.lib)
            xr, xi = x64r.float(), x64i.float()
            if rcond:
                # condition estimate from the FP64 factors narrowed to FP32
                Kr.copy_(K64r)
                Ki.copy_(K64i)
                check(self.lib.hbem_lu_rcond(N, F, _t_ptr(Kr), _t_ptr(Ki), lda, N * lda, _t_ptr(anorm), _t_ptr(rc),
                                             st), "hbem_lu_rcond", self.lib)
            del K64r, K64i
            return xr, xi, info, iters, resid, rc
        refine = _refines(mode, max_iter)
        if mode == "mixed":
            max_iter = max(1, int(max_iter))
        K0r = K0i = None
        if refine:
            K0r, K0i = Kr.clone(), Ki.clone()
        xr, xi = br.clone(), bi.clone()
        # refined plain solves factor with the TF32x3 tensor-core bulk update; the FP64-residual passes
        # recover what its 22-bit split products give away
        prec = HBEM_PREC_MIXED if mode == "mixed" else (HBEM_PREC_TF32X3 if refine else HBEM_PREC_PLAIN)
        check(self.lib.hbem_lu_factor(N, F, _t_ptr(Kr), _t_ptr(Ki), lda, N * lda, _t_ptr(piv), N, _t_ptr(info), prec,
                                      st), "hbem_lu_factor", self.lib)
        if rcond:
            check(self.lib.hbem_lu_rcond(N, F, _t_ptr(Kr), _t_ptr(Ki), lda, N * lda, _t_ptr(anorm), _t_ptr(rc), st),
                  "hbem_lu_rcond", self.lib)
        check(self.lib.hbem_lu_solve(N, 1, F, _t_ptr(Kr), _t_ptr(Ki), lda, N * lda, _t_ptr(piv), N, _t_ptr(xr),
                                     _t_ptr(xi), 1, N, HBEM_TRANS_N, st), "hbem_lu_solve", self.lib)
        if refine:
            check(self.lib.hbem_refine(N, F, _t_ptr(K0r), _t_ptr(K0i), lda, N * lda, _t_ptr(Kr), _t_ptr(Ki), N * lda,
                                       _t_ptr(piv), N, _t_ptr(br), _t_ptr(bi), N, _t_ptr(xr), _t_ptr(xi), N,
                                       float(tol), int(max_iter), _t_ptr(iters), _t_ptr(resid), st),
                  "hbem_refine", self.lib)
            del K0r, K0i
        return xr, xi, info, iters, resid, rc

    def _coupled_chunk_schur(self, k_re, k_im, kf, q, obs_t, want, mode, tol, max_iter, times, rcond=False):
        import torch

        dev, st = obs_t.device, _stream_ptr()
        F, n, m, N_obs = k_re.shape[0], self.n_dof, self.m_aperture, obs_t.shape[1]
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
        ev[0].record()
        Ar, Ai, br, bi = self.assemble(k_re, q, k_imag=k_im)
        sia_r = torch.empty((F, n, m), dtype=torch.float32, device=dev); sia_i = torch.empty_like(sia_r)
        saa_r = torch.empty((F, m, m), dtype=torch.float32, device=dev); saa_i = torch.empty_like(saa_r)
        check(self.lib.hbem_aperture_assemble(self.handle, F, _np_ptr(k_re), _np_ptr(k_im), _np_ptr(kf), _t_ptr(sia_r),
                                              _t_ptr(sia_i), _t_ptr(saa_r), _t_ptr(saa_i), st),
              "hbem_aperture_assemble", self.lib)
        minv_r = torch.empty_like(saa_r); minv_i = torch.empty_like(saa_r)
        info_ap = torch.zeros(F, dtype=torch.int32, device=dev)
        check(self.lib.hbem_coupled_ib_schur(self.handle, F, _t_ptr(Ar), _t_ptr(Ai), _t_ptr(sia_r), _t_ptr(sia_i),
                                             _t_ptr(saa_r), _t_ptr(saa_i), _t_ptr(minv_r), _t_ptr(minv_i),
                                             _t_ptr(info_ap), st), "hbem_coupled_ib_schur", self.lib)
        del sia_r, sia_i, saa_r, saa_i
        ev[1].record()
        xr, xi, info, iters, resid, rc = self._factor_solve_refine(Ar, Ai, br, bi, n, F, mode, tol, max_iter, rcond)
        del Ar, Ai
        ev[2].record()
        qa_r = torch.empty((F, m), dtype=torch.float32, device=dev); qa_i = torch.empty_like(qa_r)
        fr = torch.empty((F, N_obs), dtype=torch.float32, device=dev); fi = torch.empty_like(fr)
        check(self.lib.hbem_coupled_ib_field(self.handle, F, _np_ptr(kf), _t_ptr(xr), _t_ptr(xi), _t_ptr(minv_r),
                                             _t_ptr(minv_i), _t_ptr(obs_t), N_obs, _t_ptr(qa_r), _t_ptr(qa_i), _t_ptr(fr),
                                             _t_ptr(fi), st), "hbem_coupled_ib_field", self.lib)
        tavg = self.tag_average(xr, xi, want).cpu().numpy() if want else None
        ev[3].record()
        return self._chunk_out(ev, times, xr, xi, qa_r, qa_i, fr, fi, info, info_ap, iters, resid, tavg, rc)

    def coupled_ib_system(self, k_re, k_im, kf, q):
        """The augmented coupled system on the device: K (F, N, L) with row stride L = N rounded up to a
        multiple of 4, [0; b] (F, N), N = m + n, and the per-frequency scale alpha of the aperture
        unknowns (q_a = alpha * x[:m])."""
        torch = require_cuda()
        dev, st = torch.device("cuda", self.device), _stream_ptr()
        k_re = np.ascontiguousarray(np.atleast_1d(k_re), dtype=np.float32)
        k_im = None if k_im is None else np.ascontiguousarray(np.atleast_1d(k_im), dtype=np.float32)
        kf = np.ascontiguousarray(np.atleast_1d(kf), dtype=np.float32)
        F, n, m, T = k_re.shape[0], self.n_dof, self.m_aperture, self.n_triangles
        N = n + m
        L = (N + 3) // 4 * 4   # row stride: 16-byte aligned rows for the LU's vector paths
        Kr = torch.empty((F, N, L), dtype=torch.float32, device=dev); Ki = torch.empty_like(Kr)
        rr = torch.zeros((F, N), dtype=torch.float32, device=dev); ri = torch.zeros_like(rr)
        qr, qi = self._split_device(q, (F, T), dev)
        off_a, off_b = m * L + m, m
        check(self.lib.hbem_assemble(
            self.handle, F, _np_ptr(k_re), _np_ptr(k_im), _t_ptr(qr), _t_ptr(qi), T, None, None,
            ctypes.c_void_p(Kr.data_ptr() + 4 * off_a), ctypes.c_void_p(Ki.data_ptr() + 4 * off_a), L, N * L,
            ctypes.c_void_p(rr.data_ptr() + 4 * off_b), ctypes.c_void_p(ri.data_ptr() + 4 * off_b), N,
            HBEM_ASM_CORRECTED, st), "hbem_assemble", self.lib)
        sia_r = torch.empty((F, n, m), dtype=torch.float32, device=dev); sia_i = torch.empty_like(sia_r)
        saa_r = torch.empty((F, m, m), dtype=torch.float32, device=dev); saa_i = torch.empty_like(saa_r)
        check(self.lib.hbem_aperture_assemble(self.handle, F, _np_ptr(k_re), _np_ptr(k_im), _np_ptr(kf), _t_ptr(sia_r),
                                              _t_ptr(sia_i), _t_ptr(saa_r), _t_ptr(saa_i), st),
              "hbem_aperture_assemble", self.lib)
        alpha = torch.empty(F, dtype=torch.float32, device=dev)
        check(self.lib.hbem_coupled_ib_augment(self.handle, F, _t_ptr(sia_r), _t_ptr(sia_i), _t_ptr(saa_r),
                                               _t_ptr(saa_i), _t_ptr(Kr), _t_ptr(Ki), L, N * L, _t_ptr(alpha), st),
              "hbem_coupled_ib_augment", self.lib)
        return Kr, Ki, rr, ri, alpha

    def _coupled_chunk_augmented(self, k_re, k_im, kf, q, obs_t, want, mode, tol, max_iter, times, rcond=False):
        import torch

        dev, st = obs_t.device, _stream_ptr()
        F, n, m, N_obs = k_re.shape[0], self.n_dof, self.m_aperture, obs_t.shape[1]
        N = n + m
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
        ev[0].record()
        Kr, Ki, rr, ri, alpha = self.coupled_ib_system(k_re, k_im, kf, q)
        ev[1].record()
        xr, xi, info, iters, resid, rc = self._factor_solve_refine(Kr, Ki, rr, ri, N, F, mode, tol, max_iter, rcond)
        del Kr, Ki
        ev[2].record()
        qa_r, qa_i = (xr[:, :m] * alpha[:, None]).contiguous(), (xi[:, :m] * alpha[:, None]).contiguous()
        pr, pi = xr[:, m:].contiguous(), xi[:, m:].contiguous()
        fr = torch.empty((F, N_obs), dtype=torch.float32, device=dev); fi = torch.empty_like(fr)
        check(self.lib.hbem_coupled_ib_field(self.handle, F, _np_ptr(kf), None, None, None, None, _t_ptr(obs_t), N_obs,
                                             _t_ptr(qa_r), _t_ptr(qa_i), _t_ptr(fr), _t_ptr(fi), st),
              "hbem_coupled_ib_field", self.lib)
        tavg = self.tag_average(pr, pi, want).cpu().numpy() if want else None
        ev[3].record()
        info_ap = torch.zeros(F, dtype=torch.int32, device=dev)
        return self._chunk_out(ev, times, pr, pi, qa_r, qa_i, fr, fi, info, info_ap, iters, resid, tavg, rc)

    @staticmethod
    def _chunk_out(ev, times, pr, pi, qa_r, qa_i, fr, fi, info, info_ap, iters, resid, tavg, rc=None):
        import torch

        torch.cuda.synchronize()
        times += [ev[0].elapsed_time(ev[1]), ev[1].elapsed_time(ev[2]), ev[2].elapsed_time(ev[3])]
        cplx = lambda a, b: (a.cpu().numpy() + 1j * b.cpu().numpy()).astype(np.complex64)  # noqa: E731
        return {"field": cplx(fr, fi), "p": cplx(pr, pi), "qa": cplx(qa_r, qa_i), "info": info.cpu().numpy(),
                "info_ap": info_ap.cpu().numpy(), "iters": iters.cpu().numpy(), "resid": resid.cpu().numpy(),
                "tavg": tavg, "rcond": None if rc is None else rc.cpu().numpy()}


# Drop-in alias for the reference's session class name.
MetalNativeStandardSession = NativeSession


def torch_complex(re, im):
    import torch

    return torch.complex(re, im)


def lu_solve_f64(A_re, A_im, b_re, b_im, nrhs: int = 1):
    """Factor (F, n, n) float64 CUDA tensors with ``hbem_lu_factor_f64`` (copies: the inputs are kept) and solve
    (F, n) right-hand sides (or (F, n, nrhs)) with ``hbem_lu_solve_f64``.  Raises on a zero pivot."""
    import torch

    lib = load_library()
    F, n = int(A_re.shape[0]), int(A_re.shape[1])
    Ar, Ai = A_re.clone().contiguous(), A_im.clone().contiguous()
    xr, xi = b_re.clone().contiguous(), b_im.clone().contiguous()
    piv = torch.empty((F, n), dtype=torch.int32, device=A_re.device)
    info = torch.empty(F, dtype=torch.int32, device=A_re.device)
    st = _stream_ptr()
    check(lib.hbem_lu_factor_f64(n, F, _t_ptr(Ar), _t_ptr(Ai), n, n * n, _t_ptr(piv), n, _t_ptr(info), st),
          "hbem_lu_factor_f64", lib)
    check(lib.hbem_lu_solve_f64(n, nrhs, F, _t_ptr(Ar), _t_ptr(Ai), n, n * n, _t_ptr(piv), n, _t_ptr(xr), _t_ptr(xi),
                                nrhs, n * nrhs, HBEM_TRANS_N, st), "hbem_lu_solve_f64", lib)
    bad = info.cpu().numpy()
    if np.any(bad != 0):
        raise RuntimeError(f"hbem_lu_factor_f64: zero pivot (info {bad.tolist()})")
    return xr, xi


class ResidentSweep:
    """Device-resident batched sweep: inputs and outputs stay in HBM.

    Pre-allocates, for ``F`` frequencies on one session, the dense matrices,
    right-hand sides, pivots and field buffers, then ``run()`` issues the same
    launch sequence as ``hbem_solve_batch`` on the current stream without any
    host transfer: corrected assembly -> LU -> solve -> field -> tag averages.
    """

    def __init__(self, session: NativeSession, k_re, k_im, q, obs_3xn, tags, precision: str = "plain",
                 rcond: bool = False, refine_tolerance: float = 1e-6, refine_max_iterations: int = 10):
        torch = require_cuda()
        self.s = session
        self.lib = session.lib
        dev = torch.device("cuda", session.device)
        self.k_re = np.ascontiguousarray(np.atleast_1d(k_re), dtype=np.float32)
        self.k_im = None if k_im is None else np.ascontiguousarray(np.atleast_1d(k_im), dtype=np.float32)
        F, n, T = self.k_re.shape[0], session.n_dof, session.n_triangles
        self.F, self.n = F, n
        self.lda = ld = matrix_ld(n)
        self.q_re, self.q_im = NativeSession._split_device(q, (F, T), dev)
        self.obs = torch.as_tensor(np.ascontiguousarray(obs_3xn, dtype=np.float32), device=dev)
        self.n_obs = int(self.obs.shape[1])
        self.tags = np.ascontiguousarray(tags, dtype=np.int32)
        self.A_re = torch.empty((F, n, ld), dtype=torch.float32, device=dev)
        self.A_im = torch.empty_like(self.A_re)
        self.b_re = torch.empty((F, n), dtype=torch.float32, device=dev)
        self.b_im = torch.empty_like(self.b_re)
        self.x_re = torch.empty_like(self.b_re)
        self.x_im = torch.empty_like(self.b_re)
        self.piv = torch.empty((F, n), dtype=torch.int32, device=dev)
        self.info = torch.empty(F, dtype=torch.int32, device=dev)
        self.f_re = torch.empty((F, self.n_obs), dtype=torch.float32, device=dev)
        self.f_im = torch.empty_like(self.f_re)
        self.tag_out = torch.empty((F, max(1, self.tags.shape[0]), 2), dtype=torch.float64, device=dev)
        self.rcond = torch.empty(F, dtype=torch.float64, device=dev) if rcond else None
        self.anorm = torch.empty(F, dtype=torch.float32, device=dev) if rcond else None
        # the condition estimate runs on a second stream beside the solves, refinement and field
        self.aux = torch.cuda.Stream(device=dev, priority=0) if rcond else None
        mode = "mixed" if precision == "mixed" else "plain"
        self.refine_tol = float(refine_tolerance)
        self.refine_max = max(1, int(refine_max_iterations)) if mode == "mixed" else int(refine_max_iterations)
        self.refine = _refines(mode, refine_max_iterations)
        # as hbem_solve_batch: a refined plain sweep factors with the TF32x3 tensor-core bulk update
        self.precision = (HBEM_PREC_MIXED if mode == "mixed" else
                          HBEM_PREC_TF32X3 if self.refine else HBEM_PREC_PLAIN)
        # the assembled matrices kept for the FP64 residuals of the refinement
        self.A0_re = torch.empty_like(self.A_re) if self.refine else None
        self.A0_im = torch.empty_like(self.A_im) if self.refine else None
        self.iters = torch.zeros(F, dtype=torch.int32, device=dev)
        self.resid = torch.zeros(F, dtype=torch.float64, device=dev)

    def assemble(self, stream=None):
        n, ld = self.n, self.lda
        check(self.lib.hbem_assemble(
            self.s.handle, self.F, _np_ptr(self.k_re), _np_ptr(self.k_im), _t_ptr(self.q_re), _t_ptr(self.q_im),
            self.s.n_triangles, None, None, _t_ptr(self.A_re), _t_ptr(self.A_im), ld, n * ld, _t_ptr(self.b_re),
            _t_ptr(self.b_im), n, HBEM_ASM_CORRECTED, _stream_ptr(stream)), "hbem_assemble", self.lib)

    def factor_solve(self, stream=None):
        n, ld, st = self.n, self.lda, _stream_ptr(stream)
        self.x_re.copy_(self.b_re)
        self.x_im.copy_(self.b_im)
        if self.refine:
            self.A0_re.copy_(self.A_re)
            self.A0_im.copy_(self.A_im)
        if self.rcond is not None:
            check(self.lib.hbem_matrix_norm1(n, self.F, _t_ptr(self.A_re), _t_ptr(self.A_im), ld, n * ld,
                                             _t_ptr(self.anorm), st), "hbem_matrix_norm1", self.lib)
        check(self.lib.hbem_lu_factor(n, self.F, _t_ptr(self.A_re), _t_ptr(self.A_im), ld, n * ld, _t_ptr(self.piv), n,
                                      _t_ptr(self.info), self.precision, st), "hbem_lu_factor", self.lib)
        if self.rcond is not None:
            import torch

            main = torch.cuda.current_stream() if stream is None else stream
            self.aux.wait_stream(main)
            check(self.lib.hbem_lu_rcond(n, self.F, _t_ptr(self.A_re), _t_ptr(self.A_im), ld, n * ld,
                                         _t_ptr(self.anorm), _t_ptr(self.rcond), _stream_ptr(self.aux)),
                  "hbem_lu_rcond", self.lib)
        check(self.lib.hbem_lu_solve(n, 1, self.F, _t_ptr(self.A_re), _t_ptr(self.A_im), ld, n * ld, _t_ptr(self.piv),
                                     n, _t_ptr(self.x_re), _t_ptr(self.x_im), 1, n, HBEM_TRANS_N, st),
              "hbem_lu_solve", self.lib)
        if self.refine:
            check(self.lib.hbem_refine(
                n, self.F, _t_ptr(self.A0_re), _t_ptr(self.A0_im), ld, n * ld, _t_ptr(self.A_re), _t_ptr(self.A_im),
                n * ld, _t_ptr(self.piv), n, _t_ptr(self.b_re), _t_ptr(self.b_im), n, _t_ptr(self.x_re),
                _t_ptr(self.x_im), n, self.refine_tol, self.refine_max, _t_ptr(self.iters), _t_ptr(self.resid), st),
                "hbem_refine", self.lib)

    def field(self, stream=None):
        st = _stream_ptr(stream)
        check(self.lib.hbem_field(
            self.s.handle, self.F, _np_ptr(self.k_re), _t_ptr(self.x_re), _t_ptr(self.x_im), self.n,
            _t_ptr(self.q_re), _t_ptr(self.q_im), self.s.n_triangles, _t_ptr(self.obs), self.n_obs,
            _t_ptr(self.f_re), _t_ptr(self.f_im), self.n_obs, st), "hbem_field", self.lib)
        if self.tags.shape[0]:
            check(self.lib.hbem_reduce_tag_avg(
                self.s.handle, self.F, _t_ptr(self.x_re), _t_ptr(self.x_im), self.n, _np_ptr(self.tags),
                self.tags.shape[0], _t_ptr(self.tag_out), st), "hbem_reduce_tag_avg", self.lib)
        if self.aux is not None:
            # join the condition estimate before the next sweep overwrites the factors
            import torch

            (torch.cuda.current_stream() if stream is None else stream).wait_stream(self.aux)

    def run(self, stream=None):
        self.assemble(stream)
        self.factor_solve(stream)
        self.field(stream)
