"""Shape gradients of exterior-field objectives by the adjoint method.

No counterpart in the reference (it has no derivatives); the forward being
differentiated is the reference's P1 Neumann solve: corrected assembly
(``main.swift:3993-4133``, Duffy ``4246-4431``), dense solve, exterior field
(``main.swift:4135-4203``).

``BoundaryField.apply(vertices, problem)`` maps vertex coordinates (V, 3) to
the complex field (F, N_obs) at fixed observation points.  Its backward pass
costs one conjugate-transposed solve with the forward's LU factors plus
kernels that recompute the quadrature pair by pair (``hbem_field_adjoint``,
``hbem_field_backward``, ``hbem_assemble_backward``); dA/dX is never formed.
The Neumann data q is held fixed (the driven faces keep their orientation),
and sessions are without symmetry planes.

``SplineHorn`` drives the walls of a round horn by radial-profile spline
control points; ``directivity_objective`` is the off-axis SPL deviation
from a -6 dB / 60 degree target.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from .native import (
    HBEM_ASM_CORRECTED, HBEM_PREC_PLAIN, HBEM_TRANS_C, HBEM_TRANS_N, NativeSession, _np_ptr, _stream_ptr, _t_ptr,
    check, require_cuda,
)


def area_normals(verts_vx3: np.ndarray, tris_tx3: np.ndarray):
    """Areas (T,) and unit normals (3, T) in float64, then float32, as the geometry buffers build them."""
    p0, p1, p2 = (verts_vx3[tris_tx3[:, i]] for i in range(3))
    cross = np.cross(p1 - p0, p2 - p0)
    twice = np.linalg.norm(cross, axis=1)
    if np.any(twice <= 0.0):
        raise ValueError("a triangle has zero area after the vertex update")
    return (np.ascontiguousarray(0.5 * twice, np.float32),
            np.ascontiguousarray((cross / twice[:, None]).T, np.float32))


class ShapeProblem:
    """A P1 Neumann exterior problem whose vertices move (topology fixed).

    ``buffers``: geometry buffers of the base mesh (no symmetry plane);
    ``k_re``: (F,) float32 wavenumbers; ``q``: (F, T) complex Neumann data;
    ``obs_3xn``: (3, N) observation points.
    """

    def __init__(self, buffers, k_re, q, obs_3xn):
        torch = require_cuda()
        self.s = NativeSession(buffers, symmetry_plane=None, check_open_edges=False)
        self.lib = self.s.lib
        self.tris = np.asarray(buffers.triangles_3xm_i32, dtype=np.int64).T.copy()
        self.n, self.T, self.V = self.s.n_dof, self.s.n_triangles, int(np.asarray(buffers.vertices_3xn_f32).shape[1])
        self.k_re = np.ascontiguousarray(np.atleast_1d(k_re), dtype=np.float32)
        self.F = int(self.k_re.shape[0])
        dev = torch.device("cuda", self.s.device)
        self.dev = dev
        self.q_re, self.q_im = NativeSession._split_device(q, (self.F, self.T), dev)
        self.obs = torch.as_tensor(np.ascontiguousarray(obs_3xn, dtype=np.float32), device=dev).contiguous()
        self.n_obs = int(self.obs.shape[1])
        self.timings: dict[str, float] = {}

    def close(self):
        self.s.close()

    # -- forward --------------------------------------------------------------
    def set_vertices(self, verts_vx3: np.ndarray):
        v = np.asarray(verts_vx3, dtype=np.float64)
        areas, normals = area_normals(v, self.tris)
        v32 = np.ascontiguousarray(v.T, dtype=np.float32)
        check(self.lib.hbem_session_set_vertices(self.s.handle, _np_ptr(v32), _np_ptr(areas), _np_ptr(normals)),
              "hbem_session_set_vertices", self.lib)

    def forward(self):
        """Assemble, factor, solve and evaluate the field on the current vertices.

        Returns (field_re, field_im, state) with state holding the LU factors
        and the surface pressure for the backward pass."""
        torch = require_cuda()
        F, n, st = self.F, self.n, _stream_ptr()
        Ar = torch.empty((F, n, n), dtype=torch.float32, device=self.dev)
        Ai = torch.empty_like(Ar)
        br = torch.empty((F, n), dtype=torch.float32, device=self.dev)
        bi = torch.empty_like(br)
        check(self.lib.hbem_assemble(self.s.handle, F, _np_ptr(self.k_re), None, _t_ptr(self.q_re), _t_ptr(self.q_im),
                                     self.T, None, None, _t_ptr(Ar), _t_ptr(Ai), n, n * n, _t_ptr(br), _t_ptr(bi), n,
                                     HBEM_ASM_CORRECTED | 4, st), "hbem_assemble", self.lib)
        piv = torch.empty((F, n), dtype=torch.int32, device=self.dev)
        info = torch.empty(F, dtype=torch.int32, device=self.dev)
        check(self.lib.hbem_lu_factor(n, F, _t_ptr(Ar), _t_ptr(Ai), n, n * n, _t_ptr(piv), n, _t_ptr(info),
                                      HBEM_PREC_PLAIN, st), "hbem_lu_factor", self.lib)
        check(self.lib.hbem_lu_solve(n, 1, F, _t_ptr(Ar), _t_ptr(Ai), n, n * n, _t_ptr(piv), n, _t_ptr(br), _t_ptr(bi),
                                     1, n, HBEM_TRANS_N, st), "hbem_lu_solve", self.lib)
        fr = torch.empty((F, self.n_obs), dtype=torch.float32, device=self.dev)
        fi = torch.empty_like(fr)
        check(self.lib.hbem_field(self.s.handle, F, _np_ptr(self.k_re), _t_ptr(br), _t_ptr(bi), n, _t_ptr(self.q_re),
                                  _t_ptr(self.q_im), self.T, _t_ptr(self.obs), self.n_obs, _t_ptr(fr), _t_ptr(fi),
                                  self.n_obs, st), "hbem_field", self.lib)
        return fr, fi, {"lu_re": Ar, "lu_im": Ai, "piv": piv, "info": info, "p_re": br, "p_im": bi}

    # -- backward -------------------------------------------------------------
    def backward(self, g_re, g_im, state):
        """dL/dX (3, V) float64 on the device for g = dL/dRe F + i dL/dIm F (F, N_obs)."""
        torch = require_cuda()
        F, n, st = self.F, self.n, _stream_ptr()
        g_re, g_im = g_re.contiguous(), g_im.contiguous()
        lam_re = torch.empty((F, n), dtype=torch.float32, device=self.dev)
        lam_im = torch.empty_like(lam_re)
        check(self.lib.hbem_field_adjoint(self.s.handle, F, _np_ptr(self.k_re), _t_ptr(self.obs), self.n_obs,
                                          _t_ptr(g_re), _t_ptr(g_im), self.n_obs, _t_ptr(lam_re), _t_ptr(lam_im), n,
                                          st), "hbem_field_adjoint", self.lib)
        check(self.lib.hbem_lu_solve(n, 1, F, _t_ptr(state["lu_re"]), _t_ptr(state["lu_im"]), n, n * n,
                                     _t_ptr(state["piv"]), n, _t_ptr(lam_re), _t_ptr(lam_im), 1, n, HBEM_TRANS_C, st),
              "hbem_lu_solve", self.lib)
        grad = torch.zeros((3, self.V), dtype=torch.float64, device=self.dev)
        check(self.lib.hbem_field_backward(self.s.handle, F, _np_ptr(self.k_re), _t_ptr(self.obs), self.n_obs,
                                           _t_ptr(g_re), _t_ptr(g_im), self.n_obs, _t_ptr(state["p_re"]),
                                           _t_ptr(state["p_im"]), n, _t_ptr(self.q_re), _t_ptr(self.q_im), self.T,
                                           _t_ptr(grad), st), "hbem_field_backward", self.lib)
        check(self.lib.hbem_assemble_backward(self.s.handle, F, _np_ptr(self.k_re), None, _t_ptr(lam_re),
                                              _t_ptr(lam_im), n, _t_ptr(state["p_re"]), _t_ptr(state["p_im"]), n,
                                              _t_ptr(self.q_re), _t_ptr(self.q_im), self.T, _t_ptr(grad), st),
              "hbem_assemble_backward", self.lib)
        return grad


def _autograd_function():
    import torch

    class BoundaryField(torch.autograd.Function):
        """vertices (V, 3) float64 -> complex64 field (F, N_obs); backward by the adjoint."""

        @staticmethod
        def forward(ctx, verts, problem: ShapeProblem):
            problem.set_vertices(verts.detach().cpu().numpy())
            fr, fi, state = problem.forward()
            if int(state["info"].abs().sum()) != 0:
                raise RuntimeError("zero pivot in the forward solve")
            ctx.problem, ctx.state = problem, state
            ctx.vdev, ctx.vdtype = verts.device, verts.dtype
            return torch.complex(fr, fi)

        @staticmethod
        def backward(ctx, g):
            g = g.to(torch.complex64)
            grad = ctx.problem.backward(g.real, g.imag, ctx.state)
            return grad.T.to(device=ctx.vdev, dtype=ctx.vdtype), None

    return BoundaryField


_BF = None


def boundary_field(verts, problem: ShapeProblem):
    """Differentiable field of ``problem`` at vertex coordinates ``verts`` (V, 3) float64 tensor."""
    global _BF
    if _BF is None:
        _BF = _autograd_function()
    return _BF.apply(verts, problem)


# ------------------------------------------------------------------ spline-driven round horn
@dataclass
class SplineHorn:
    """Round horn whose flare walls move radially by a cubic B-spline of the axial coordinate.

    Wall vertices with 0 < z < L move by dr(z) = sin(pi z / L) sum_k c_k B_k(z / L)
    along their radial direction (inner and outer walls together, so the lip
    thickness is kept); the throat disc, can and lip stay.  ``c`` (metres) are
    the control points.
    """

    base: np.ndarray          # (V, 3) float64 base vertices
    basis: np.ndarray         # (V, K) float64: dr = basis @ c
    radial: np.ndarray        # (V, 3) unit radial directions (0 for fixed vertices)

    def vertices(self, c):
        """Vertex coordinates (V, 3) for control points ``c`` (torch tensor or numpy array)."""
        try:
            import torch

            if isinstance(c, torch.Tensor):
                b = torch.as_tensor(self.basis, dtype=c.dtype, device=c.device)
                rad = torch.as_tensor(self.radial, dtype=c.dtype, device=c.device)
                base = torch.as_tensor(self.base, dtype=c.dtype, device=c.device)
                return base + (b @ c)[:, None] * rad
        except ImportError:  # pragma: no cover
            pass
        c = np.asarray(c, dtype=np.float64)
        return self.base + (self.basis @ c)[:, None] * self.radial


def bspline_basis(u: np.ndarray, n_ctrl: int, degree: int = 3) -> np.ndarray:
    """Clamped uniform B-spline basis (len(u), n_ctrl) by the Cox-de Boor recursion."""
    n_knots = n_ctrl + degree + 1
    inner = np.linspace(0.0, 1.0, n_knots - 2 * degree)
    knots = np.concatenate([np.zeros(degree), inner, np.ones(degree)])
    u = np.clip(np.asarray(u, dtype=np.float64), 0.0, 1.0 - 1e-12)
    B = np.zeros((u.size, n_knots - 1))
    for i in range(n_knots - 1):
        B[:, i] = (knots[i] <= u) & (u < knots[i + 1])
    for d in range(1, degree + 1):
        nb = np.zeros((u.size, n_knots - 1 - d))
        for i in range(n_knots - 1 - d):
            den1 = knots[i + d] - knots[i]
            den2 = knots[i + d + 1] - knots[i + 1]
            t1 = (u - knots[i]) / den1 * B[:, i] if den1 > 0 else 0.0
            t2 = (knots[i + d + 1] - u) / den2 * B[:, i + 1] if den2 > 0 else 0.0
            nb[:, i] = t1 + t2
        B = nb
    return B[:, :n_ctrl]


def spline_horn(spec, n_ctrl: int = 24):
    """(LoadedMesh, SplineHorn) for the full (no symmetry) horn of ``spec``."""
    from . import generators as G

    mesh = G.horn(spec, quarter=False)
    v = np.asarray(mesh.grid.vertices, dtype=np.float64).T.copy()
    z = v[:, 2]
    rho = np.hypot(v[:, 0], v[:, 1])
    L = spec.length
    move = (z > 1e-9) & (z < L - 1e-9) & (rho > 1e-9)
    u = np.where(move, z / L, 0.0)
    basis = bspline_basis(u, n_ctrl) * (np.sin(np.pi * u) * move)[:, None]
    radial = np.zeros_like(v)
    radial[move, 0] = v[move, 0] / rho[move]
    radial[move, 1] = v[move, 1] / rho[move]
    return mesh, SplineHorn(base=v, basis=basis, radial=radial)


def directivity_points(mouth_z: float, angles_deg, distance: float = 2.0) -> np.ndarray:
    """(3, 1 + 2 A): the on-axis point, then the angles in the xz plane, then in the yz plane."""
    pts = [(0.0, 0.0, mouth_z + distance)]
    for plane in (0, 1):
        for a in angles_deg:
            t = np.deg2rad(a)
            p = [0.0, 0.0, mouth_z + distance * np.cos(t)]
            p[plane] = distance * np.sin(t)
            pts.append(tuple(p))
    return np.asarray(pts, dtype=np.float64).T


def directivity_objective(field, angles_deg, slope_db_per_deg: float = -6.0 / 60.0):
    """sum_f sum_(plane, angle) (SPL(angle) - SPL(0) - slope * angle)^2 for ``field`` (F, 1 + 2 A).

    Works on torch tensors (differentiable) and numpy arrays."""
    try:
        import torch

        if isinstance(field, torch.Tensor):
            mag = field.abs().to(torch.float64)
            rel = 20.0 * torch.log10(mag[:, 1:] / mag[:, :1])
            tgt = torch.as_tensor(np.tile(slope_db_per_deg * np.asarray(angles_deg, np.float64), 2),
                                  device=rel.device)
            return ((rel - tgt[None, :]) ** 2).sum()
    except ImportError:  # pragma: no cover
        pass
    mag = np.abs(np.asarray(field))
    rel = 20.0 * np.log10(mag[:, 1:] / mag[:, :1])
    tgt = np.tile(slope_db_per_deg * np.asarray(angles_deg, np.float64), 2)
    return float(((rel - tgt[None, :]) ** 2).sum())
