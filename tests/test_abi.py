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
