"""Batched, graph-captured sweeps over meshes of different sizes and symmetry
against per-mesh eager sweeps through the same C ABI (same kernels: equal to
FP32 rounding of the variant's summation order)."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import golden_buffers

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a CUDA device", allow_module_level=True)

from hornlab_metal_bem_b200.batch import CANDIDATES, BatchedSweeps, SweepCase  # noqa: E402
from hornlab_metal_bem_b200.native import NativeSession, ResidentSweep  # noqa: E402

CASES = [("horn_quarter", "yz+xz", (900.0, 4000.0, 9000.0)), ("ico2", None, (300.0, 1200.0)),
         ("yz_half", "yz", (500.0, 2500.0, 6000.0, 11000.0))]


def _cases():
    out = []
    rng = np.random.default_rng(3)
    for name, plane, freqs in CASES:
        b = golden_buffers(name)
        T = b.triangles_3xm_i32.shape[1]
        k = (2 * np.pi * np.asarray(freqs) / 343.0).astype(np.float32)
        q = np.zeros((len(freqs), T), np.complex64)
        q[:, b.physical_tags_i32 == b.physical_tags_i32.max()] = 1.2041
        q[:, ::7] += (rng.normal(size=(len(freqs), len(range(0, T, 7)))) * 0.1).astype(np.complex64)
        obs = np.array([[0.0, 0.8, 1.5], [0.0, 0.3, 0.2], [2.0, 1.5, 0.5]], np.float32)
        tags = sorted({int(t) for t in np.unique(b.physical_tags_i32)})
        out.append(SweepCase(b, k, q, obs, tags, plane))
    return out


def _eager(case):
    with NativeSession(case.buffers, symmetry_plane=case.symmetry_plane, check_open_edges=False) as s:
        rs = ResidentSweep(s, case.k_re, None, case.q, case.obs, case.tags)
        rs.run()
        torch.cuda.synchronize()
        f = rs.f_re.cpu().numpy() + 1j * rs.f_im.cpu().numpy()
        t = rs.tag_out.cpu().numpy()
        return f, t[..., 0] + 1j * t[..., 1]


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("tuning", [None, {"n<=768": CANDIDATES[4], "n<=1536": CANDIDATES[2]}, "auto"])
def test_batched_graph_sweeps_match_eager(tuning, tmp_path):
    cases = _cases()
    ref = [_eager(c) for c in cases]
    kw = {"cache_path": tmp_path / "tune.json"} if tuning == "auto" else {}
    bs = BatchedSweeps(cases, n_streams=2, tuning=tuning, **kw)
    try:
        for _ in range(2):   # replays reuse the slot workspaces
            bs.run()
        outs = bs.outputs()
    finally:
        bs.close()
    tol = 1e-5 if tuning is None else 1e-4
    for (f_ref, t_ref), o, c in zip(ref, outs, cases):
        assert np.all(o.lapack_info == 0)
        assert o.field.shape == (len(c.k_re), c.obs.shape[1])
        assert _rel(o.field, f_ref) < tol
        assert _rel(o.tag_average, t_ref) < tol
    if tuning == "auto":
        assert (tmp_path / "tune.json").exists()
