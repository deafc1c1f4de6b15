"""Structured errors with stable codes (mirrors src/lunarscout/errors.py:7-154
for the classes the horizon and lighting facades raise)."""

from __future__ import annotations

from collections.abc import Mapping
from typing import Any


class LunarscoutError(Exception):
    """Base class of structured errors: ``code`` and ``details``."""

    default_code = "lunarscout_error"

    def __init__(self, message: str, *, code: str | None = None,
                 details: Mapping[str, Any] | None = None) -> None:
        super().__init__(message)
        self.code = str(code or self.default_code)
        self.details = dict(details or {})


class InputError(LunarscoutError):
    default_code = "input_error"


class HorizonError(LunarscoutError):
    default_code = "horizon_error"


class HorizonFormatError(HorizonError):
    default_code = "horizon_format_error"


class HorizonGenerationError(HorizonError):
    default_code = "horizon_generation_error"


class ComputeBackendError(LunarscoutError):
    default_code = "compute_backend_error"


class CudaError(ComputeBackendError):
    default_code = "cuda_error"


class ProductError(LunarscoutError):
    default_code = "product_error"


class ProductCalculationError(ProductError):
    default_code = "product_calculation_error"


class OperationCancelledError(LunarscoutError):
    default_code = "operation_cancelled"


def is_cuda_runtime_failure(error: BaseException) -> bool:
    """True when the exception (or its cause chain) comes from the CUDA stack:
    its type's module is ``cuda`` / ``cuda.*`` (ls/horizon.py:29-40)."""
    seen: set[int] = set()
    current: BaseException | None = error
    while current is not None and id(current) not in seen:
        seen.add(id(current))
        module = type(current).__module__.lower()
        if module == "cuda" or module.startswith(("cuda.", "numba.cuda")):
            return True
        current = current.__cause__ or current.__context__
    return False
