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


def _c3_case(seed: int, freqs_hz):
    """One of the batching workload's seeded half (yz) waveguides at a few of its frequencies."""
    import hornlab_metal_bem_b200 as hb
    from hornlab_metal_bem_b200 import generators as G
    from hornlab_metal_bem_b200.bie import build_source_face_scale
    from hornlab_metal_bem_b200.geometry import build_geometry_buffers
    from hornlab_metal_bem_b200.mesh import make_pure_function_spaces
    from hornlab_metal_bem_b200.observation import build_observation_points
    from hornlab_metal_bem_b200.sweep import field_points_3xn, k_values, neumann_rows

    cfg = hb.native_config(freq_min_hz=500.0, freq_max_hz=20000.0, freq_count=40, source_motion="axial",
                           native_symmetry_plane="yz", native_check_open_edges=False,
                           observation=hb.ObservationConfig(planes=["horizontal", "vertical", "diagonal"],
                                                            angle_count=37))
    spec = G.horn_spec_from_seed(seed, edge=343.0 / 8000.0 / 6.0, flare_range=(10.0, 40.0),
                                 mouth_range=(0.080, 0.200))
    mesh = G.horn(spec, quarter=False, half=True)
    frame = hb._resolve_frame(mesh, cfg)
    obs, _ = build_observation_points(frame, cfg.observation)
    p1, dp0 = make_pure_function_spaces(mesh.grid)
    buf = build_geometry_buffers(mesh.grid, mesh.physical_tags, p1, dp0)
    freqs = np.asarray(freqs_hz, np.float64)
    k_re, _ = k_values(freqs, cfg)
    scale = build_source_face_scale(mesh.grid, mesh.physical_tags, cfg, frame.axis, frame.source_center)
    q = neumann_rows(buf.n_triangles, mesh.physical_tags, freqs, cfg, scale)
    return SweepCase(buf, k_re, q, field_points_3xn(obs), sorted(cfg.velocity_sources), "yz")


def _db(z):
    return 20 * np.log10(np.abs(z))


def test_batched_sweeps_match_oracle_on_waveguide_batch_meshes():
    """The two smallest meshes of the 64-waveguide batch (seeds 43 and 0: 829 and 866 dofs), captured and
    replayed with the device-side refinement, against the FP64 oracle (oracle assembly, LAPACK zgesv,
    oracle field and tag averages) across the band, 20 kHz included."""
    from oracle.oracle import Oracle, dense_solve

    cases = [_c3_case(43, (2000.0, 12000.0, 20000.0)), _c3_case(0, (700.0, 16000.0))]
    bs = BatchedSweeps(cases, n_streams=2, tuning=None)
    try:
        bs.run()
        bs.run()
        outs = bs.outputs()
    finally:
        bs.close()
    for c, o in zip(cases, outs):
        assert c.n in (829, 866)
        assert np.all(o.lapack_info == 0)
        assert np.all((o.refine_iterations >= 0) & (o.refine_iterations <= 3))
        assert np.all(o.refine_residual_rel < 1e-5)
        orc = Oracle(c.buffers, 1, "f64")
        for f in range(len(c.k_re)):
            A, b = orc.corrected(float(c.k_re[f]), c.q[f], 0.0, None)
            p = dense_solve(A, b, "f64")
            fld = orc.field(float(c.k_re[f]), p, c.q[f].astype(np.complex128), c.obs)
            assert _rel(o.field[f], fld) < 1e-4, (c.n, f)
            assert np.max(np.abs(_db(o.field[f]) - _db(fld))) < 0.01
            for t, tag in enumerate(c.tags):
                ref = orc.tag_average(p, tag)
                assert abs(o.tag_average[f, t] - ref) <= 1e-4 * abs(ref), (c.n, f, tag)
