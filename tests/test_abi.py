"""The C ABI: libhbem.so loads, exports every entry point of include/hbem.h and
rejects bad arguments before touching a device (no compute calls here)."""
from __future__ import annotations

import ctypes
import re
import subprocess

import pytest

from conftest import REPO

from hornlab_metal_bem_b200 import native


def _declared_functions() -> list[str]:
    text = (REPO / "include" / "hbem.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:int|long long)\s+(hbem_\w+)\s*\(", text, flags=re.M)))


def test_library_exports_every_declared_symbol():
    lib_path = native.LIB_PATH
    assert lib_path.exists(), "run python -m hornlab_metal_bem_b200.csrc.build"
    out = subprocess.run(["nm", "-D", "--defined-only", str(lib_path)], capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r"\bT (hbem_\w+)", out))
    declared = _declared_functions()
    assert len(declared) >= 12
    missing = [f for f in declared if f not in exported]
    assert not missing, missing
    lib = native.load_library()
    for name in declared:
        assert getattr(lib, name) is not None
    assert set(native._SIGNATURES) == set(declared)


def test_version_and_error_channel():
    lib = native.load_library()
    assert lib.hbem_version() >= 100
    out = ctypes.c_void_p()
    rc = lib.hbem_session_create(None, 0, None, 0, None, 0, None, None, None, 0, 0, ctypes.byref(out))
    assert rc == -1
    assert "NULL geometry" in native.last_error(lib)
    rc = lib.hbem_lu_factor(4, 1, None, None, 4, 16, None, 4, None, 0, None)
    assert rc == -1 and "NULL pointer" in native.last_error(lib)
    rc = lib.hbem_session_query(None, 0, None)
    assert rc == -1


def test_session_requires_cuda_without_fallback(monkeypatch):
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is visible")
    from conftest import golden_buffers

    with pytest.raises(native.BackendUnavailable):
        native.NativeSession(golden_buffers("tiny"))


def test_tuning_knobs_validate_and_read_back():
    """hbem_set_tuning accepts each knob's documented values (0 = built-in choice), rejects the rest with a
    message naming the knob, and hbem_get_tuning reads the value back; host-only, no device needed."""
    lib = native.load_library()
    text = (REPO / "include" / "hbem.h").read_text()
    keys = {m.group(1): int(m.group(2)) for m in re.finditer(r"#define (HBEM_TUNE_\w+) (\d+)", text)}
    count = keys.pop("HBEM_TUNE_COUNT")
    assert sorted(keys.values()) == list(range(count))
    valid = {
        "HBEM_TUNE_ASM_MINBLOCKS": ([0, 2, 3], [1, 4]),
        "HBEM_TUNE_LU_PANEL": ([0, 16, 32, 64], [8, 48, 128]),
        "HBEM_TUNE_LU_SOLVE": ([0, 1, 2, 3], [-1, 4]),
        "HBEM_TUNE_ASM_PAIRS": ([0, 1], [2]),
        "HBEM_TUNE_DUFFY": ([0, 1, 2], [3]),
        "HBEM_TUNE_LU_LOOKAHEAD": ([0, 1], [2]),
        "HBEM_TUNE_LU_RESERVE": ([0, 1, 17, 1024], [-1, 1025]),
        "HBEM_TUNE_WAVE_SPIN": ([0, 1, 4194304], [-1, 4194305]),
        "HBEM_TUNE_LU_UPDATE": ([0, 1, 2], [-1, 3]),
        "HBEM_TUNE_LU_BLOCK": ([0, 32, 64, 128], [16, 256, -1]),
        "HBEM_TUNE_LU_PANEL_KERNEL": ([0, 1], [-1, 2]),
    }
    assert set(valid) == set(keys)
    try:
        for name, key in keys.items():
            ok, bad = valid[name]
            for v in ok:
                assert lib.hbem_set_tuning(key, v) == 0, (name, v)
                assert lib.hbem_get_tuning(key) == v
            for v in bad:
                assert lib.hbem_set_tuning(key, v) == -1, (name, v)
                assert name in native.last_error(lib)
                assert lib.hbem_get_tuning(key) == ok[-1]   # a rejected value changes nothing
        assert lib.hbem_set_tuning(count, 0) == -1
        assert "unknown key" in native.last_error(lib)
    finally:
        for key in keys.values():
            lib.hbem_set_tuning(key, 0)


def test_entry_points_validate_arguments_before_any_device_work():
    """Every rejection below happens on the host, before a device is touched (this runs without one):
    status -1 (HBEM_ERR_ARG) and a message naming the entry point; empty problems are no-ops."""
    import numpy as np

    lib = native.load_library()
    D = ctypes.c_void_p(256)          # a non-NULL pointer the checks never dereference
    err = lambda: native.last_error(lib)

    # empty problems succeed without looking at any pointer
    assert lib.hbem_lu_factor(0, 1, None, None, 1, 1, None, 1, None, 0, None) == 0
    assert lib.hbem_lu_solve(4, 1, 0, None, None, 4, 16, None, 4, None, None, 1, 4, 0, None) == 0
    assert lib.hbem_refine(4, 0, None, None, 4, 16, None, None, 16, None, 4, None, None, 4, None, None, 4,
                           1e-6, 3, None, None, None) == 0
    # factor: strides, precision
    assert lib.hbem_lu_factor(4, 1, D, D, 3, 16, D, 4, D, 0, None) == -1 and "bad strides" in err()
    assert lib.hbem_lu_factor(4, 1, D, D, 4, 12, D, 4, D, 0, None) == -1 and "bad strides" in err()
    assert lib.hbem_lu_factor(4, 1, D, D, 4, 16, D, 4, D, 2, None) == -1 and "precision" in err()
    # solve: NULL, strides, transposition
    assert lib.hbem_lu_solve(4, 1, 1, D, D, 4, 16, None, 4, D, D, 1, 4, 0, None) == -1 and "NULL" in err()
    assert lib.hbem_lu_solve(4, 1, 1, D, D, 4, 16, D, 3, D, D, 1, 4, 0, None) == -1 and "bad strides" in err()
    assert lib.hbem_lu_solve(4, 1, 1, D, D, 4, 16, D, 4, D, D, 1, 4, 3, None) == -1 and "trans" in err()
    # refinement: tolerance and iteration count
    args = (4, 1, D, D, 4, 16, D, D, 16, D, 4, D, D, 4, D, D, 4)
    assert lib.hbem_refine(*args, 0.0, 3, None, None, None) == -1 and "hbem_refine" in err()
    assert lib.hbem_refine(*args, 1e-6, -1, None, None, None) == -1 and "hbem_refine" in err()
    assert lib.hbem_refine_noalloc(*args, float("nan"), 3, None, None, None) == -1 and "noalloc" in err()
    assert lib.hbem_refine_async(*args, 1e-6, -2, None, None, None) == -1 and "async" in err()
    assert lib.hbem_refine_async(4, 1, D, D, 4, 16, D, D, 15, D, 4, D, D, 4, D, D, 4, 1e-6, 2, None, None,
                                 None) == -1 and "too small" in err()
    # condition estimate: strides and the largest order its shared-memory vector holds
    assert lib.hbem_matrix_norm1(4, 1, D, D, 4, 15, D, None) == -1 and "bad strides" in err()
    n = 30000
    assert lib.hbem_lu_rcond(n, 1, D, D, n, n * n, D, D, None) == -1 and "too large" in err()
    # batch sweep without a session
    assert lib.hbem_solve_batch(None, 1, *([None] * 5), 0, None, 0, 0, 1e-6, 0, *([None] * 11)) == -1
    assert "NULL session" in err()

    # session creation: geometry checks run before the device is queried
    v = np.ascontiguousarray(np.array([[0.0, 1, 0, 0], [0, 0, 1, 0], [0, 0, 0, 1]], np.float32))
    t = np.ascontiguousarray(np.array([[0, 0, 0, 1], [2, 1, 3, 2], [1, 3, 2, 3]], np.int32))
    l2g = np.ascontiguousarray(t.T)
    tags = np.array([1, 1, 1, 2], np.int32)
    areas = np.full(4, 0.5, np.float32)
    normals = np.ascontiguousarray(np.zeros((3, 4), np.float32))
    P = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    out = ctypes.c_void_p()

    def create(v=v, t=t, l2g=l2g, areas=areas, n_dof=4, sym=0):
        return lib.hbem_session_create(P(v), v.shape[1], P(t), t.shape[1], P(l2g), n_dof, P(tags), P(areas),
                                       P(normals), sym, 0, ctypes.byref(out))

    assert create(sym=5) == -1 and "sym_code" in err()
    bad_t = t.copy()
    bad_t[0, 0] = 7
    assert create(t=bad_t) == -1 and "vertex index out of range" in err()
    bad_l2g = l2g.copy()
    bad_l2g[0, 0] = 4
    assert create(l2g=bad_l2g) == -1 and "out-of-range DOF" in err()
    bad_areas = areas.copy()
    bad_areas[2] = 0.0
    assert create(areas=bad_areas) == -1 and "non-positive area" in err()
    assert create(n_dof=0) == -1 and "empty geometry" in err()
