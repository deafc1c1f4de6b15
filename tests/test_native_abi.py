"""The C-ABI library loads and exports every declared symbol (no GPU calls)."""

from __future__ import annotations

import ctypes
import re
import subprocess
import sys

import pytest

from conftest import ROOT

HEADERS = sorted((ROOT / "include").glob("*.h"))


def declared_functions() -> list[str]:
    names = []
    for header in HEADERS:
        text = header.read_text()
        names += re.findall(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(ls200_\w+)\s*\(", text, re.M)
    return sorted(set(names))


def test_headers_declare_entry_points():
    names = declared_functions()
    assert "ls200_march_all_passes" in names
    assert "ls200_context_create" in names
    assert len(names) >= 15


def test_library_exports_every_declared_symbol():
    from lunarscout_b200 import _native

    library = ctypes.CDLL(str(_native.LIBRARY_PATH))
    missing = [name for name in declared_functions() if not hasattr(library, name)]
    assert not missing, missing


def test_python_binding_covers_every_declared_symbol():
    from lunarscout_b200 import _native

    _native.library()
    assert set(declared_functions()) <= set(_native.SIGNATURES)


def declared_arities() -> dict[str, int]:
    """Parameter count of every declaration in include/*.h."""
    arities = {}
    for header in HEADERS:
        text = re.sub(r"/\*.*?\*/", "", header.read_text(), flags=re.S)
        for name, params in re.findall(
                r"\b(?:ls200_status|int|const char \*)\s*(ls200_\w+)\s*\(([^;]*?)\)\s*;", text,
                flags=re.S):
            params = params.strip()
            arities[name] = 0 if params in ("", "void") else params.count(",") + 1
    return arities


def test_python_argument_lists_match_the_header():
    from lunarscout_b200 import _native

    arities = declared_arities()
    assert set(arities) == set(declared_functions())
    mismatched = {name: (count, len(_native.SIGNATURES[name]))
                  for name, count in arities.items()
                  if len(_native.SIGNATURES[name]) != count}
    assert not mismatched, mismatched


def test_import_does_not_initialise_cuda():
    code = (
        "import sys; sys.path.insert(0, %r)\n"
        "import lunarscout_b200, lunarscout_b200.cuda_backend, lunarscout_b200._native\n"
        "import ctypes.util\n"
        "print('torch' in sys.modules)\n"
    ) % str(ROOT)
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True,
                         check=True)
    assert out.stdout.strip() == "False"


def test_no_device_raises_cuda_backend_error():
    """Without a visible sm_100 device the session refuses to start."""
    try:
        import torch

        if torch.cuda.is_available():
            pytest.skip("a GPU is visible")
    except ImportError:
        pass
    from lunarscout_b200.cuda_backend import CudaBackendError, CudaSession

    with pytest.raises(CudaBackendError):
        CudaSession(0)


def test_execution_error_is_classified_as_cuda_failure():
    """lunarscout maps exceptions whose type module starts with 'cuda.' to
    cuda_*_execution_failed (ls/horizon.py:29-40)."""
    from lunarscout_b200._native import CudaExecutionError

    assert type(CudaExecutionError("x")).__module__.startswith("cuda.")


def test_status_codes_map_to_reference_exceptions(monkeypatch):
    from lunarscout_b200 import _native

    monkeypatch.setattr(_native, "last_error", lambda: "boom")
    with pytest.raises(ValueError):
        _native.check(_native.LS200_ERR_INVALID)
    with pytest.raises(_native.CudaBackendError):
        _native.check(_native.LS200_ERR_UNAVAILABLE)
    with pytest.raises(_native.CudaExecutionError):
        _native.check(_native.LS200_ERR_CUDA)
    with pytest.raises(_native.CudaTimeoutError):
        _native.check(_native.LS200_ERR_TIMEOUT)
    _native.check(_native.LS200_OK)
