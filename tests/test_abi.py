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
