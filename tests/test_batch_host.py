"""Host logic of batched sweeps: stream assignment, size buckets, the autotuner's choice and cache."""
from __future__ import annotations

import json

from hornlab_metal_bem_b200.batch import CANDIDATES, Autotuner, lpt_slots, size_bucket


def test_lpt_slots_balances_and_covers_every_job():
    costs = [9.0, 7.0, 6.0, 5.0, 4.0, 3.0, 1.0]
    slots = lpt_slots(costs, 3)
    assert sorted(i for s in slots for i in s) == list(range(len(costs)))
    loads = [sum(costs[i] for i in s) for s in slots]
    assert max(loads) - min(loads) <= max(costs)
    assert lpt_slots(costs, 1) == [[0, 1, 2, 3, 4, 5, 6]]
    assert len(lpt_slots([1.0, 2.0], 8)) == 2


def test_size_buckets_are_monotone():
    names = [size_bucket(n) for n in (100, 768, 769, 1536, 2000, 3072, 5000, 7000)]
    assert names == ["n<=768", "n<=768", "n<=1536", "n<=1536", "n<=3072", "n<=3072", "n<=6144", "n>6144"]


class _Case:
    def __init__(self, n):
        self.n = n


def test_autotuner_picks_fastest_per_bucket_and_caches(tmp_path):
    calls = []

    def timer(case, variant):
        calls.append((case.n, dict(variant)))
        # small meshes prefer the 16-wide panel, large ones the 3-CTA assembly
        if case.n <= 768:
            return 1.0 if variant["panel"] == 16 else 2.0
        return 1.0 if variant["asm"] == 3 else 2.0

    cache = tmp_path / "tune.json"
    cases = [_Case(n) for n in (500, 600, 700, 2000, 2500)]
    t = Autotuner(timer, "gpu-x|1", cache)
    table = t.tune(cases)
    assert table["n<=768"]["panel"] == 16
    assert table["n<=3072"]["asm"] == 3
    assert len(calls) == 2 * len(CANDIDATES)
    # the representative of a bucket is its median-size case
    assert {c[0] for c in calls} == {600, 2500}
    assert json.loads(cache.read_text())["gpu-x|1"] == table
    # a second tuner on the same GPU reads the cache and times nothing
    calls.clear()
    t2 = Autotuner(timer, "gpu-x|1", cache)
    assert t2.tune(cases) == table and not calls
    assert t2.variant_for(650)["panel"] == 16
    # another GPU model tunes afresh
    t3 = Autotuner(timer, "gpu-y|1", cache)
    t3.tune(cases)
    assert len(calls) == 2 * len(CANDIDATES)
    assert set(json.loads(cache.read_text())) == {"gpu-x|1", "gpu-y|1"}


def test_matrix_pitch_and_solve_names():
    """The sweep paths' dense row pitch is n rounded up to 4 floats (16-byte rows), and a refined plain
    solve is reported as the FP32 LU with the TF32x3 tensor-core bulk."""
    from hornlab_metal_bem_b200.native import matrix_ld, solve_impl

    assert [matrix_ld(n) for n in (1, 4, 1043, 1044, 18749)] == [4, 4, 1044, 1044, 18752]
    assert solve_impl("plain", False) == "hbem_blocked_lu_fp32"
    assert solve_impl("plain", True) == "hbem_blocked_lu_fp32_tf32x3_refined"
    assert solve_impl("mixed", True) == "hbem_blocked_lu_bf16x3_refined"
    assert solve_impl("fp64", False) == "hbem_blocked_lu_fp64"
