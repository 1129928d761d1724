"""Batched frequency sweeps over many meshes of uneven size.

No counterpart in the reference, which runs one mesh per session and one
helper process per operation.  Here every (mesh, frequency) case of a batch
stays on the device:

* each mesh's sweep (corrected assembly -> LU -> solve -> FP64-residual
  refinement -> field -> tag averages over all its frequencies) is captured
  once into a CUDA graph and replayed, so its hundreds of launches cost one
  graph launch (the refinement decides its stopping rule on the device);
* meshes are spread over a few streams by longest-processing-time order of
  their estimated cost (n^3 for the LU, T^2 M for the assembly), so small
  meshes overlap with large ones; meshes on one stream share one workspace
  sized for the largest of them;
* an autotuner picks, per mesh-size bucket, the kernel variants (ordered or
  unordered pair assembly and its occupancy, Duffy wavenumbers per warp, LU
  sub-panel width, solve scheme) by timing candidates on a
  representative mesh, and caches the choice per GPU model.
"""
from __future__ import annotations

import json
import os
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

from .native import (
    HBEM_ASM_CORRECTED, HBEM_PREC_PLAIN, HBEM_PREC_TF32X3, HBEM_TRANS_N, NativeSession, _np_ptr, _stream_ptr, _t_ptr,
    check, load_library, matrix_ld, require_cuda,
)

TUNE_ASM_MINBLOCKS, TUNE_LU_PANEL, TUNE_LU_SOLVE, TUNE_ASM_PAIRS, TUNE_DUFFY = 0, 1, 2, 3, 4
IMAGES = {None: 1, "yz": 2, "xz": 2, "yz+xz": 4, "xy": 2}


@dataclass(eq=False)
class SweepCase:
    """One mesh and its frequency sweep (inputs of ``assemble_solve_evaluate``)."""

    buffers: object
    k_re: np.ndarray                 # (F,) float32
    q: np.ndarray                    # (F, T) complex Neumann data
    obs: np.ndarray                  # (3, N) observation points
    tags: list = field(default_factory=list)
    symmetry_plane: str | None = None
    k_im: np.ndarray | None = None

    @property
    def n(self) -> int:
        return int(self.buffers.p1_dof_count)

    @property
    def T(self) -> int:
        return int(self.buffers.triangles_3xm_i32.shape[1])

    def cost(self) -> float:
        """Relative device time: LU (8/3 n^3 / ~25 TFLOP/s) + assembly (36 T^2 M / ~1e12 samples/s), per frequency."""
        F = len(self.k_re)
        return F * ((8.0 / 3.0) * self.n ** 3 / 25e12 + 36.0 * self.T ** 2 * IMAGES[self.symmetry_plane] / 1e12)


@dataclass
class CaseOutput:
    field: np.ndarray                # (F, N) complex64
    tag_average: np.ndarray          # (F, n_tags) complex128
    lapack_info: np.ndarray          # (F,) int
    surface_pressure: np.ndarray | None = None
    refine_iterations: np.ndarray | None = None     # (F,) refinement passes applied
    refine_residual_rel: np.ndarray | None = None   # (F,) ||b - A x|| / ||b|| after them (0 without refinement)


def lpt_slots(costs, n_slots: int) -> list[list[int]]:
    """Longest-processing-time assignment of jobs to ``n_slots`` streams (each slot keeps descending cost order)."""
    n_slots = max(1, min(int(n_slots), len(costs))) if len(costs) else 1
    load = [0.0] * n_slots
    slots: list[list[int]] = [[] for _ in range(n_slots)]
    for i in sorted(range(len(costs)), key=lambda j: -costs[j]):
        s = min(range(n_slots), key=lambda j: load[j])
        slots[s].append(i)
        load[s] += costs[i]
    return slots


def size_bucket(n: int) -> str:
    for lim in (768, 1536, 3072, 6144):
        if n <= lim:
            return f"n<={lim}"
    return "n>6144"


# ------------------------------------------------------------------ autotuner
CANDIDATES = (
    {"asm": 0, "panel": 0, "solve": 0, "pairs": 0, "duffy": 0},
    {"asm": 0, "panel": 0, "solve": 0, "pairs": 1, "duffy": 0},
    {"asm": 3, "panel": 0, "solve": 0, "pairs": 1, "duffy": 0},
    {"asm": 0, "panel": 16, "solve": 0, "pairs": 0, "duffy": 0},
    {"asm": 0, "panel": 0, "solve": 1, "pairs": 0, "duffy": 0},
    {"asm": 0, "panel": 0, "solve": 0, "pairs": 0, "duffy": 1},
)


def default_cache_path() -> Path:
    env = os.environ.get("HBEM_AUTOTUNE_CACHE")
    if env:
        return Path(env)
    return Path(os.path.expanduser("~")) / ".cache" / "hornlab_metal_bem_b200" / "autotune.json"


class Autotuner:
    """Per size bucket, the fastest candidate variant for a sweep.

    ``timer(case, variant) -> seconds`` measures one sweep of ``case`` with
    ``variant`` applied; the choice is cached under ``device_key`` (GPU
    model) in a JSON file.
    """

    def __init__(self, timer, device_key: str, cache_path: Path | None = None, candidates=CANDIDATES):
        self.timer = timer
        self.device_key = device_key
        self.cache_path = Path(cache_path) if cache_path is not None else default_cache_path()
        self.candidates = list(candidates)
        self.table: dict[str, dict] = {}
        self.measurements: dict[str, list] = {}
        self._load()

    def _load(self):
        try:
            data = json.loads(self.cache_path.read_text())
            self.table = dict(data.get(self.device_key, {}))
        except (OSError, ValueError):
            self.table = {}

    def _save(self):
        try:
            data = json.loads(self.cache_path.read_text()) if self.cache_path.exists() else {}
        except (OSError, ValueError):
            data = {}
        data[self.device_key] = self.table
        try:
            self.cache_path.parent.mkdir(parents=True, exist_ok=True)
            self.cache_path.write_text(json.dumps(data, indent=1, sort_keys=True))
        except OSError:
            pass

    def variant_for(self, n: int) -> dict:
        return dict(self.table.get(size_bucket(n), self.candidates[0]))

    def tune(self, cases, force: bool = False) -> dict[str, dict]:
        """Time every candidate on the median-size case of each bucket not yet in the table."""
        by_bucket: dict[str, list] = {}
        for c in cases:
            by_bucket.setdefault(size_bucket(c.n), []).append(c)
        changed = False
        for b, cs in sorted(by_bucket.items()):
            if b in self.table and not force:
                continue
            rep = sorted(cs, key=lambda c: c.n)[len(cs) // 2]
            times = [(float(self.timer(rep, v)), i) for i, v in enumerate(self.candidates)]
            best = min(times)[1]
            self.table[b] = dict(self.candidates[best])
            self.measurements[b] = [{"variant": self.candidates[i], "seconds": t} for t, i in times]
            changed = True
        if changed:
            self._save()
        return dict(self.table)


def apply_variant(lib, variant: dict) -> None:
    check(lib.hbem_set_tuning(TUNE_ASM_MINBLOCKS, int(variant.get("asm", 0))), "hbem_set_tuning", lib)
    check(lib.hbem_set_tuning(TUNE_LU_PANEL, int(variant.get("panel", 0))), "hbem_set_tuning", lib)
    check(lib.hbem_set_tuning(TUNE_LU_SOLVE, int(variant.get("solve", 0))), "hbem_set_tuning", lib)
    check(lib.hbem_set_tuning(TUNE_ASM_PAIRS, int(variant.get("pairs", 0))), "hbem_set_tuning", lib)
    check(lib.hbem_set_tuning(TUNE_DUFFY, int(variant.get("duffy", 0))), "hbem_set_tuning", lib)


# ------------------------------------------------------------------ batched runner
class _Slot:
    """One stream and the workspace shared by the meshes assigned to it."""

    def __init__(self, torch, dev, n_max: int, F_max: int, refine: bool):
        self.stream = torch.cuda.Stream(device=dev)
        self.A_re = torch.empty((F_max, n_max, matrix_ld(n_max)), dtype=torch.float32, device=dev)
        self.A_im = torch.empty_like(self.A_re)
        # the assembled matrices, kept for the FP64 residuals of the refinement
        self.A0_re = torch.empty_like(self.A_re) if refine else None
        self.A0_im = torch.empty_like(self.A_re) if refine else None
        self.b_re = torch.empty((F_max, n_max), dtype=torch.float32, device=dev)
        self.b_im = torch.empty_like(self.b_re)
        self.x_re = torch.empty_like(self.b_re)
        self.x_im = torch.empty_like(self.b_re)
        self.piv = torch.empty((F_max, n_max), dtype=torch.int32, device=dev)


class _CaseRun:
    """Device inputs / outputs of one case and its launch sequence."""

    def __init__(self, torch, dev, case: SweepCase, write_surface_pressure: bool, refine_tolerance: float,
                 refine_max_iterations: int):
        self.case = case
        self.refine_tol = float(refine_tolerance)
        self.refine_max = int(refine_max_iterations)
        self.s = NativeSession(case.buffers, symmetry_plane=case.symmetry_plane, check_open_edges=False)
        self.lib = self.s.lib
        F, T = len(case.k_re), case.T
        self.F, self.n = F, self.s.n_dof
        self.k_re = np.ascontiguousarray(case.k_re, dtype=np.float32)
        self.k_im = None if case.k_im is None else np.ascontiguousarray(case.k_im, dtype=np.float32)
        self.q_re, self.q_im = NativeSession._split_device(case.q, (F, T), dev)
        self.obs = torch.as_tensor(np.ascontiguousarray(case.obs, dtype=np.float32), device=dev).contiguous()
        self.n_obs = int(self.obs.shape[1])
        self.tags_h = np.ascontiguousarray(case.tags, dtype=np.int32)
        self.tags = torch.as_tensor(self.tags_h, device=dev)
        self.info = torch.empty(F, dtype=torch.int32, device=dev)
        self.iters = torch.zeros(F, dtype=torch.int32, device=dev)
        self.resid = torch.zeros(F, dtype=torch.float64, device=dev)
        self.f_re = torch.empty((F, self.n_obs), dtype=torch.float32, device=dev)
        self.f_im = torch.empty_like(self.f_re)
        self.tag_out = torch.zeros((F, max(1, len(case.tags)), 2), dtype=torch.float64, device=dev)
        self.p_re = torch.empty((F, self.n), dtype=torch.float32, device=dev) if write_surface_pressure else None
        self.p_im = torch.empty_like(self.p_re) if write_surface_pressure else None
        self.graph = None

    def launch(self, slot: _Slot):
        """The sweep's launches on the current stream (captured or eager)."""
        n, F, st, lib, s = self.n, self.F, _stream_ptr(), self.lib, self.s
        ld = matrix_ld(n)   # rows on 16-byte boundaries
        A_re, A_im = slot.A_re.view(-1)[:F * n * ld], slot.A_im.view(-1)[:F * n * ld]
        b_re, b_im = slot.b_re.view(-1)[:F * n], slot.b_im.view(-1)[:F * n]
        x_re, x_im = slot.x_re.view(-1)[:F * n], slot.x_im.view(-1)[:F * n]
        piv = slot.piv.view(-1)[:F * n]
        check(lib.hbem_assemble(s.handle, F, _np_ptr(self.k_re), _np_ptr(self.k_im), _t_ptr(self.q_re),
                                _t_ptr(self.q_im), s.n_triangles, None, None, _t_ptr(A_re), _t_ptr(A_im), ld, n * ld,
                                _t_ptr(b_re), _t_ptr(b_im), n, HBEM_ASM_CORRECTED | 4, st), "hbem_assemble", lib)
        x_re.copy_(b_re)
        x_im.copy_(b_im)
        if self.refine_max > 0:
            A0_re, A0_im = slot.A0_re.view(-1)[:F * n * ld], slot.A0_im.view(-1)[:F * n * ld]
            A0_re.copy_(A_re)
            A0_im.copy_(A_im)
        # refined sweeps factor with the TF32x3 tensor-core bulk update (the refinement recovers FP32 accuracy)
        prec = HBEM_PREC_TF32X3 if self.refine_max > 0 else HBEM_PREC_PLAIN
        check(lib.hbem_lu_factor(n, F, _t_ptr(A_re), _t_ptr(A_im), ld, n * ld, _t_ptr(piv), n, _t_ptr(self.info),
                                 prec, st), "hbem_lu_factor", lib)
        check(lib.hbem_lu_solve(n, 1, F, _t_ptr(A_re), _t_ptr(A_im), ld, n * ld, _t_ptr(piv), n, _t_ptr(x_re),
                                _t_ptr(x_im), 1, n, HBEM_TRANS_N, st), "hbem_lu_solve", lib)
        if self.refine_max > 0:
            check(lib.hbem_refine_async(n, F, _t_ptr(A0_re), _t_ptr(A0_im), ld, n * ld, _t_ptr(A_re), _t_ptr(A_im),
                                        n * ld, _t_ptr(piv), n, _t_ptr(b_re), _t_ptr(b_im), n, _t_ptr(x_re),
                                        _t_ptr(x_im), n, self.refine_tol, self.refine_max, _t_ptr(self.iters),
                                        _t_ptr(self.resid), st), "hbem_refine_async", lib)
        check(lib.hbem_field(s.handle, F, _np_ptr(self.k_re), _t_ptr(x_re), _t_ptr(x_im), n, _t_ptr(self.q_re),
                             _t_ptr(self.q_im), s.n_triangles, _t_ptr(self.obs), self.n_obs, _t_ptr(self.f_re),
                             _t_ptr(self.f_im), self.n_obs, st), "hbem_field", lib)
        if len(self.tags_h):
            check(lib.hbem_reduce_tag_avg_device(s.handle, F, _t_ptr(x_re), _t_ptr(x_im), n, _t_ptr(self.tags),
                                                 len(self.tags_h), _t_ptr(self.tag_out), st),
                  "hbem_reduce_tag_avg_device", lib)
        if self.p_re is not None:
            self.p_re.view(-1).copy_(x_re)
            self.p_im.view(-1).copy_(x_im)

    def output(self) -> CaseOutput:
        f = (self.f_re.cpu().numpy() + 1j * self.f_im.cpu().numpy()).astype(np.complex64)
        t = self.tag_out.cpu().numpy()
        tav = (t[..., 0] + 1j * t[..., 1])[:, :len(self.tags_h)]
        sp = None
        if self.p_re is not None:
            sp = (self.p_re.cpu().numpy() + 1j * self.p_im.cpu().numpy()).astype(np.complex64)
        return CaseOutput(field=f, tag_average=tav, lapack_info=self.info.cpu().numpy(), surface_pressure=sp,
                          refine_iterations=self.iters.cpu().numpy(), refine_residual_rel=self.resid.cpu().numpy())


class BatchedSweeps:
    """All frequencies of many meshes, graph-captured per mesh, on ``n_streams`` concurrent streams.

    ``tuning``: "auto" (autotune per size bucket, cached), None (built-in
    variants) or a dict bucket -> variant.  Call ``run()`` any number of
    times; ``outputs()`` copies the last results to the host.  Each FP32 LU
    solution is refined with FP64 residuals (``hbem_refine_async``: at most
    ``refine_max_iterations`` passes, stopping at ``refine_tolerance`` or when
    a pass no longer lowers the residual; 0 keeps the unrefined cgesv result).
    """

    def __init__(self, cases: list[SweepCase], n_streams: int = 4, tuning="auto", cache_path=None,
                 write_surface_pressure: bool = False, use_graphs: bool = True, refine_tolerance: float = 1e-6,
                 refine_max_iterations: int = 3):
        torch = require_cuda()
        self.torch = torch
        self.lib = load_library()
        self.dev = torch.device("cuda", torch.cuda.current_device())
        self.cases = list(cases)
        self.runs = [_CaseRun(torch, self.dev, c, write_surface_pressure, refine_tolerance, refine_max_iterations)
                     for c in self.cases]
        costs = [c.cost() for c in self.cases]
        self.slot_of_case: dict[int, int] = {}
        self.slot_cases = lpt_slots(costs, n_streams)
        self.slots = []
        for si, members in enumerate(self.slot_cases):
            n_max = max(self.runs[i].n for i in members)
            F_max = max(self.runs[i].F for i in members)
            self.slots.append(_Slot(torch, self.dev, n_max, F_max, refine_max_iterations > 0))
            for i in members:
                self.slot_of_case[i] = si
        self.autotuner = None
        self.variants: dict[int, dict] = {}
        if tuning == "auto":
            name = torch.cuda.get_device_name(self.dev)
            self.autotuner = Autotuner(self._time_case, f"{name}|{self._version()}", cache_path)
            self.autotuner.tune(self.cases)
            self.variants = {i: self.autotuner.variant_for(c.n) for i, c in enumerate(self.cases)}
        elif isinstance(tuning, dict):
            self.variants = {i: dict(tuning.get(size_bucket(c.n), CANDIDATES[0])) for i, c in enumerate(self.cases)}
        else:
            self.variants = {i: dict(CANDIDATES[0]) for i in range(len(self.cases))}
        self.use_graphs = use_graphs
        if use_graphs:
            self._capture()
        apply_variant(self.lib, CANDIDATES[0])

    def _version(self) -> str:
        return str(int(self.lib.hbem_version()))

    def _time_case(self, case: SweepCase, variant: dict) -> float:
        torch = self.torch
        i = next(j for j, c in enumerate(self.cases) if c is case)
        run, slot = self.runs[i], self.slots[self.slot_of_case[i]]
        apply_variant(self.lib, variant)
        with torch.cuda.stream(slot.stream):
            run.launch(slot)                       # warm-up (module set-up, caches)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(2):
                run.launch(slot)
            e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) * 1e-3 / 2

    def _capture(self):
        torch = self.torch
        for i, run in enumerate(self.runs):
            slot = self.slots[self.slot_of_case[i]]
            apply_variant(self.lib, self.variants[i])
            with torch.cuda.stream(slot.stream):
                run.launch(slot)                   # eager run first: one-time set-up stays out of the graph
            torch.cuda.synchronize()
            g = torch.cuda.CUDAGraph()
            before = int(self.lib.hbem_launch_count())
            with torch.cuda.graph(g, stream=slot.stream, capture_error_mode="relaxed"):
                run.launch(slot)
            run.graph = g
            run.graph_kernels = int(self.lib.hbem_launch_count()) - before
        torch.cuda.synchronize()

    def run(self):
        """Every case once, slots concurrently; returns when all are queued (not synchronised)."""
        torch = self.torch
        cur = torch.cuda.current_stream()
        for slot in self.slots:
            slot.stream.wait_stream(cur)
        for si, members in enumerate(self.slot_cases):
            slot = self.slots[si]
            with torch.cuda.stream(slot.stream):
                for i in members:
                    if self.use_graphs:
                        self.runs[i].graph.replay()
                    else:
                        apply_variant(self.lib, self.variants[i])
                        self.runs[i].launch(slot)
        for slot in self.slots:
            cur.wait_stream(slot.stream)

    def kernels_per_run(self) -> int:
        """Kernels of this library one ``run()`` launches (graph nodes counted at capture)."""
        return sum(getattr(r, "graph_kernels", 0) for r in self.runs)

    def set_neumann(self, q_list) -> int:
        """Copy new Neumann data (host (F, T) complex per case) into the captured input buffers; returns bytes."""
        nbytes = 0
        for run, q in zip(self.runs, q_list):
            q = np.asarray(q).reshape(run.F, run.case.T)
            re = self.torch.from_numpy(np.ascontiguousarray(q.real, dtype=np.float32)).pin_memory()
            im = self.torch.from_numpy(np.ascontiguousarray(q.imag, dtype=np.float32)).pin_memory()
            run.q_re.copy_(re, non_blocking=True)
            run.q_im.copy_(im, non_blocking=True)
            nbytes += 8 * q.size
        return nbytes

    def outputs(self) -> list[CaseOutput]:
        self.torch.cuda.synchronize()
        return [r.output() for r in self.runs]

    def close(self):
        for r in self.runs:
            r.graph = None
            r.s.close()
