"""Generate the golden fixtures under tests/golden/ from the reference's own Python.

Run where a checkout of the reference is available, naming its root:

    python tests/golden/make_golden.py --reference <path to the hornlab-metal-bem checkout>

It imports ``hornlab_metal_bem`` (and the fixture helpers of the reference's
``tests/test_metal_native.py``) from that checkout, evaluates the front-end
functions of the hot path and the FP64 subdivided-quadrature pair helper on
small seeded inputs, and stores inputs + outputs as ``.npz``.  The tests
compare this package against these files; nothing reads the reference at
test time.
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import sys
from pathlib import Path
from types import SimpleNamespace

import numpy as np

OUT = Path(__file__).resolve().parent
REPO = OUT.parent.parent


def _load_reference(ref: Path):
    sys.path.insert(0, str(ref))
    import hornlab_metal_bem  # noqa: F401
    from hornlab_metal_bem import bie, observation, sweep
    from hornlab_metal_bem.config import (
        AnnularProfile,
        AxialProfile,
        ObservationConfig,
        PerFaceProfile,
        SolveConfig,
        TaperProfile,
    )
    from hornlab_metal_bem.metal import geometry

    spec = importlib.util.spec_from_file_location("ref_test_metal_native", ref / "tests" / "test_metal_native.py")
    tmod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(tmod)
    return SimpleNamespace(
        bie=bie, obs=observation, sweep=sweep, geometry=geometry, tmod=tmod,
        SolveConfig=SolveConfig, ObservationConfig=ObservationConfig,
        AxialProfile=AxialProfile, TaperProfile=TaperProfile, AnnularProfile=AnnularProfile,
        PerFaceProfile=PerFaceProfile,
    )


def _meshes():
    sys.path.insert(0, str(REPO))
    from hornlab_metal_bem_b200 import generators as G

    out = {
        "ico2": G.icosphere(2, 0.1),
        "horn_quarter": G.horn(G.HornSpec(edge=0.014), quarter=True),
        "horn_full": G.horn(G.HornSpec(edge=0.016, flare=30.0, lip=0.004), quarter=False),
    }
    return out


def _buffers_dict(prefix, b):
    return {
        f"{prefix}vertices": b.vertices_3xn_f32,
        f"{prefix}triangles": b.triangles_3xm_i32,
        f"{prefix}tags": b.physical_tags_i32,
        f"{prefix}l2g": b.p1_local2global_i32,
        f"{prefix}areas": b.triangle_areas_f32,
        f"{prefix}normals": b.triangle_normals_3xm_f32,
        f"{prefix}p1_count": np.int64(b.p1_dof_count),
    }


def _near_pairs(buffers, count: int) -> list[tuple[int, int]]:
    """Deterministic near, non-touching (test, trial) pairs: scanning test triangles in order, the nearest
    triangle that shares no vertex, kept when its centroid distance is under 1.5 x the larger diameter."""
    v = np.asarray(buffers.vertices_3xn_f32, dtype=np.float64)
    tri = np.asarray(buffers.triangles_3xm_i32)
    pts = v[:, tri]                                  # (3 coords, 3 vertices, T)
    cen = pts.mean(axis=1)
    diam = np.max([np.linalg.norm(pts[:, i] - pts[:, j], axis=0) for i in range(3) for j in range(3)], axis=0)
    out = []
    for t in range(tri.shape[1]):
        ratio = np.linalg.norm(cen - cen[:, [t]], axis=0) / np.maximum(diam, diam[t])
        for s_ in np.argsort(ratio):
            if s_ == t or set(tri[:, t]) & set(tri[:, s_]):
                continue
            if ratio[s_] < 1.5:
                out.append((int(t), int(s_)))
            break
        if len(out) == count:
            break
    return out


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True, help="root of the hornlab-metal-bem checkout")
    args = ap.parse_args()
    R = _load_reference(Path(args.reference))
    meshes = _meshes()
    known: dict = {}

    # 1. geometry buffers: reference test fixtures + generated meshes
    geo: dict = {}
    fixtures = {
        "tiny": R.tmod._tiny_geometry_buffers,
        "near": R.tmod._near_quadrature_geometry_buffers,
        "ib_box": R.tmod._ib_box_geometry_buffers,
        "ib_quarter_box": R.tmod._ib_quarter_box_geometry_buffers,
        "ib_quarter_box_full": R.tmod._ib_quarter_box_mirrored_full_geometry_buffers,
        "yzxz_quarter": R.tmod._tiny_yz_xz_parity_quarter_buffers,
        "yzxz_full": R.tmod._tiny_yz_xz_full_buffers,
        "yzxz_quarter_multi": R.tmod._tiny_yz_xz_quarter_buffers,
        "yz_half": R.tmod._tiny_yz_parity_half_buffers,
        "yz_full": R.tmod._tiny_yz_full_buffers,
        "xy_half": R.tmod._tiny_xy_parity_half_buffers,
        "xy_full": R.tmod._tiny_xy_full_buffers,
    }
    for name, fn in fixtures.items():
        geo.update(_buffers_dict(f"{name}__", fn()))
    for name, m in meshes.items():
        from hornlab_metal_bem.mesh import make_pure_function_spaces

        p1, dp0 = make_pure_function_spaces(m.grid)
        b = R.geometry.build_metal_geometry_buffers(m.grid, m.physical_tags, p1, dp0)
        geo.update(_buffers_dict(f"{name}__", b))
        geo[f"{name}__in_vertices"] = np.asarray(m.grid.vertices)
        geo[f"{name}__in_elements"] = np.asarray(m.grid.elements)
        geo[f"{name}__in_tags"] = np.asarray(m.physical_tags)
    np.savez_compressed(OUT / "geometry.npz", **geo)

    # symmetry validation verdicts on the reference fixtures
    verdicts = {}
    for name, plane, check in (
        ("yzxz_quarter", "yz+xz", False), ("yzxz_quarter_multi", "yz+xz", True),
        ("yz_half", "yz", False), ("xy_half", "xy", False), ("tiny", "yz", True), ("ib_quarter_box", "yz+xz", True),
    ):
        try:
            R.geometry.validate_native_symmetry_plane(fixtures[name](), plane, check_open_edges=check)
            verdicts[f"{name}|{plane}|{check}"] = "ok"
        except Exception as exc:  # noqa: BLE001
            verdicts[f"{name}|{plane}|{check}"] = type(exc).__name__
    for name, tag, plane in (("ib_box", 7, None), ("ib_quarter_box", 7, "yz+xz"), ("tiny", 2, None)):
        try:
            R.geometry.validate_native_infinite_baffle_aperture(fixtures[name](), tag, symmetry_plane=plane)
            verdicts[f"aperture|{name}|{tag}|{plane}"] = "ok"
        except Exception as exc:  # noqa: BLE001
            verdicts[f"aperture|{name}|{tag}|{plane}"] = type(exc).__name__
    known["validation_verdicts"] = verdicts

    # 2. frames and observation points
    fr: dict = {}
    frame_cases = [
        ("ico2", 2, "mouth", None), ("ico2", 2, "throat", None),
        ("horn_quarter", 2, "mouth", "yz+xz"), ("horn_quarter", 2, "throat", "yz+xz"),
        ("horn_full", 2, "mouth", None), ("horn_full", 1, "mouth", None),
    ]
    for i, (name, tag, origin, plane) in enumerate(frame_cases):
        m = meshes[name]
        f = R.obs.infer_frame(m.grid, m.physical_tags, source_tag=tag, origin_at=origin, symmetry_plane=plane)
        for key in ("axis", "origin", "u", "v", "mouth_center", "source_center"):
            fr[f"{i}__{key}"] = getattr(f, key)
        oc = R.ObservationConfig(planes=["horizontal", "vertical", "diagonal"], distance_m=2.0, angle_count=37)
        pts, ang = R.obs.build_observation_points(f, oc)
        fr[f"{i}__points"] = pts
        fr[f"{i}__angles"] = ang
    known["frame_cases"] = frame_cases
    np.savez_compressed(OUT / "frames.npz", **fr)

    # 3. Neumann rows
    nm: dict = {}
    full = meshes["horn_full"]
    from hornlab_metal_bem.mesh import make_pure_function_spaces

    p1, dp0 = make_pure_function_spaces(full.grid)
    frame = R.obs.infer_frame(full.grid, full.physical_tags, source_tag=2)
    n_src = int(np.sum(full.physical_tags == 2))
    rng = np.random.default_rng(7)
    perface = rng.normal(size=n_src) + 1j * rng.normal(size=n_src)
    neumann_cases = {
        "vel_normal": dict(velocity_mode="velocity"),
        "acc_normal": dict(velocity_mode="acceleration"),
        "vel_axial": dict(velocity_mode="velocity", source_motion="axial"),
        "acc_taper": dict(velocity_mode="acceleration", source_velocity_profiles={2: R.TaperProfile("raised_cosine", 0.5)}),
        "vel_taper_lin": dict(velocity_mode="velocity", source_velocity_profiles={2: R.TaperProfile("linear", 0.3)}),
        "vel_annular": dict(velocity_mode="velocity", source_velocity_profiles={2: R.AnnularProfile(0.2, 0.8)}),
        "vel_perface": dict(velocity_mode="velocity", source_velocity_profiles={2: R.PerFaceProfile(perface)}),
        "vel_two_tags": dict(velocity_mode="velocity", velocity_sources={2: 1.0, 1: 0.25}, air_density=1.205),
        "robin_skip": dict(velocity_mode="velocity", velocity_sources={2: 1.0, 1: 0.5}, impedance_sources={1: 0.3 + 0.1j}),
    }
    freqs = np.array([250.0, 1234.5, 9000.0])
    for name, kw in neumann_cases.items():
        cfg = R.SolveConfig(**kw)
        scale = R.bie._build_source_face_scale(full.grid, full.physical_tags, cfg, frame.axis, frame.source_center)
        imp = R.sweep._impedance_sources_for_frequencies(full.physical_tags, freqs, cfg)
        rows = R.sweep._build_neumann_rows(dp0, full.physical_tags, freqs, cfg, imp, source_face_scale=scale)
        nm[f"{name}__rows"] = rows
        k_re, k_im = R.sweep._k_values_for_native(freqs, cfg)
        nm[f"{name}__k"] = k_re
    nm["freqs"] = freqs
    nm["perface"] = perface
    known["neumann_cases"] = list(neumann_cases)
    np.savez_compressed(OUT / "neumann.npz", **nm)

    # 4. directivity + reductions
    rd: dict = {}
    p = rng.normal(size=(4, 3, 37)) + 1j * rng.normal(size=(4, 3, 37))
    p[1, 0, 5] = 0.0
    rd["pressure"] = p
    rd["directivity"] = np.stack([R.sweep._directivity_from_pressure(p[i], 0) for i in range(4)])
    rd["directivity_idx3"] = np.stack([R.sweep._directivity_from_pressure(p[i], 3) for i in range(4)])
    ps = rng.normal(size=p1.global_dof_count) + 1j * rng.normal(size=p1.global_dof_count)
    rd["surface"] = ps
    surf = SimpleNamespace(coefficients=ps)
    rd["impedance_tag2"] = R.bie._compute_impedance(full.grid, surf, full.physical_tags, p1, source_tag=2)
    pav = R.bie.compute_surface_pressure_avg(full.grid, surf, full.physical_tags, p1, [1, 2, 9])
    rd["pavg"] = np.array([pav[1], pav[2], pav[9]])
    np.savez_compressed(OUT / "reductions.npz", **rd)

    # 5. FP64 subdivided-quadrature pair blocks (reference test helper, level 4)
    pb: dict = {}
    near = R.tmod._near_quadrature_geometry_buffers()
    cases = [("near", 0, 1, 1.8318326), ("near", 1, 0, 9.0)]
    ico = meshes["ico2"]
    p1i, dp0i = make_pure_function_spaces(ico.grid)
    icob = R.geometry.build_metal_geometry_buffers(ico.grid, ico.physical_tags, p1i, dp0i)
    tris = icob.triangles_3xm_i32.T
    picks = []
    for t in range(tris.shape[0]):
        if len(set(tris[0]) & set(tris[t])) == 0 and len(picks) < 3 and t > 5:
            picks.append(t)
    cases += [("ico2", 0, t, 18.3) for t in picks]
    # near but not touching pairs: for each triangle in turn, the closest triangle sharing no vertex
    # (centroid distance under 1.5 times the larger diameter), on the sphere and on the quarter horn
    # (whose folded lip brings walls close together)
    built = {"ico2": icob}
    for name, count in (("ico2", 2), ("horn_quarter", 4)):
        if name not in built:
            m = meshes[name]
            p1m, dp0m = make_pure_function_spaces(m.grid)
            built[name] = R.geometry.build_metal_geometry_buffers(m.grid, m.physical_tags, p1m, dp0m)
        cases += [(name, t, s_, 18.3) for t, s_ in _near_pairs(built[name], count)]
    for i, (name, test, trial, k) in enumerate(cases):
        b = near if name == "near" else built[name]
        ref = R.tmod._reference_pair_blocks(b, test, trial, k, 4)
        pb[f"{i}__slp"] = ref.slp
        pb[f"{i}__dlp"] = ref.dlp
    known["pair_block_cases"] = cases
    np.savez_compressed(OUT / "pair_blocks.npz", **pb)

    # 6. known answers from the reference tests (read as text there)
    known["tiny_pair_plan"] = {"coincident": 2, "edge": 2, "vertex": 0, "unique_triplets": 16}
    known["yzxz_quarter_image_adjacent_pairs"] = 15
    (OUT / "known_answers.json").write_text(json.dumps(known, indent=1, default=str), encoding="utf-8")
    print("wrote", sorted(p.name for p in OUT.iterdir()))


if __name__ == "__main__":
    main()
