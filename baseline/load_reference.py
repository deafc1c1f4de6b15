"""Import the reference lunarscout installed under ``baseline/_ref``.

The reference is installed unmodified with ``pip install --no-deps --target
baseline/_ref``.  Its top-level ``lunarscout/__init__`` needs
pyproj, rasterio and spiceypy, which this image does not have, so the
hot-path modules are imported through a stub ``lunarscout`` package whose
path is the installed source; nothing of the reference is copied or edited.

``enable_numba_cuda`` replaces the reference's import gate
(``lunarscout/_cuda_runtime.py:12``, which insists on the separate
``numba-cuda`` distribution) with numba's built-in CUDA target, so the
reference's own ``CudaSession`` can run on the GPU.

Used by the benchmark's reference legs and by the drop-in tests that run the
reference's pipeline with this project's sessions swapped in; the product
never imports it.
"""

from __future__ import annotations

import importlib
import os
import sys
import tempfile
import types
from pathlib import Path

INSTALL = Path(__file__).resolve().parent / "_ref"
PACKAGE = INSTALL / "lunarscout"


def available() -> bool:
    """Whether the reference is installed here."""
    return (PACKAGE / "_numba_horizon" / "cuda_backend.py").is_file()


def import_reference(*, enable_numba_cuda: bool = False) -> types.ModuleType:
    """Return the reference's ``lunarscout._numba_horizon`` package."""
    if not available():
        raise ModuleNotFoundError(f"the reference is not installed under {INSTALL}")
    os.environ.setdefault("NUMBA_CACHE_DIR",
                          str(Path(tempfile.gettempdir()) / "lunarscout-reference-numba"))
    existing = sys.modules.get("lunarscout")
    if existing is None:
        stub = types.ModuleType("lunarscout")
        stub.__path__ = [str(PACKAGE)]
        sys.modules["lunarscout"] = stub
    elif list(getattr(existing, "__path__", [])) != [str(PACKAGE)]:
        raise ImportError("another lunarscout package is already imported")
    if enable_numba_cuda:
        runtime = importlib.import_module("lunarscout._cuda_runtime")

        def import_numba_cuda():
            import numba
            from numba import cuda

            return numba, cuda

        runtime.import_numba_cuda = import_numba_cuda
    return importlib.import_module("lunarscout._numba_horizon")


def module(name: str) -> types.ModuleType:
    """A module of the reference package, e.g. ``module("_numba_horizon.pipeline")``."""
    import_reference()
    return importlib.import_module(f"lunarscout.{name}")
