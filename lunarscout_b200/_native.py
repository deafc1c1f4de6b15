"""ctypes binding of ``libls200.so`` (the C ABI declared in include/ls200.h).

Loading the library does not initialise CUDA; only creating a context does.
There is no fallback: if the library is missing or no sm_100 device is usable,
callers get :class:`CudaBackendError`, and a failing kernel or copy raises
:class:`CudaExecutionError`.
"""

from __future__ import annotations

import ctypes
import threading
import weakref
from pathlib import Path

import numpy as np

LIBRARY_PATH = Path(__file__).resolve().parent / "libls200.so"

LS200_OK = 0
LS200_ERR_INVALID = 1
LS200_ERR_CUDA = 2
LS200_ERR_UNAVAILABLE = 3
LS200_ERR_TIMEOUT = 4


class CudaBackendError(RuntimeError):
    """The CUDA backend is unavailable (mirrors cuda_backend.py:19-20)."""


class CudaExecutionError(RuntimeError):
    """A CUDA call failed while executing.

    Its module name starts with ``cuda.`` so that lunarscout's public error
    mapping (ls/horizon.py:29-40, ls/products.py:73-84) classifies it as a
    CUDA execution failure, exactly as it does for Numba-CUDA errors.
    """


CudaExecutionError.__module__ = "cuda.ls200"


class CudaTimeoutError(CudaExecutionError):
    """A bounded device wait gave up and the kernel returned early."""


CudaTimeoutError.__module__ = "cuda.ls200"

_lib = None
_lock = threading.Lock()

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")
_vp = ctypes.c_void_p
_i = ctypes.c_int
_i64 = ctypes.c_int64
_d = ctypes.c_double
_f = ctypes.c_float

# name -> argtypes (restype is always int status unless listed in _RESTYPES)
SIGNATURES: dict[str, list] = {
    "ls200_last_error": [],
    "ls200_abi_version": [],
    "ls200_context_create": [_i, _vp],
    "ls200_context_destroy": [_vp],
    "ls200_device_info": [_vp, ctypes.c_char_p, _i, _vp, _vp, _vp],
    "ls200_set_stream": [_vp, _vp],
    "ls200_reset_stream": [_vp],
    "ls200_synchronize": [_vp],
    "ls200_pyramid_layout": [_i, _i, _vp, _i, _vp, _vp],
    "ls200_build_max_pyramid": [_vp, _f32p, _i, _i, _f32p],
    "ls200_dem_create": [_vp, _f32p, _i, _i, _vp, _f64p, _f64p, _f32p, _vp],
    "ls200_dem_destroy": [_vp],
    "ls200_dem_download_mips": [_vp, _f32p, _i64],
    "ls200_segments": [_vp, _vp, _i, _i, _i, _i, _i, _d, _d, _i, _f32p],
    "ls200_segments_device": [_vp, _vp, _i, _i, _i, _i, _i, _d, _d, _i, _vp],
    "ls200_march_pass": [_vp, _f32p, _i, _i, _i, _vp, _vp, _i, _i, _i, _i, _i, _i, _f,
                         _vp, _f32p],
    "ls200_march_all_passes": [_vp, _f32p, _i, _i, _i, _vp, _i, _i, _i, _i, _i, _f, _f32p,
                               _vp],
    "ls200_march_all_passes_device": [_vp, _vp, _i, _i, _i, _vp, _i, _i, _i, _i, _i, _f,
                                      _vp, _i, _vp],
    "ls200_set_counting": [_vp, _i],
    "ls200_last_counters": [_vp, _vp, _vp, _vp],
    "ls200_slopes_to_degrees": [_vp, _f32p, _i64, _f32p],
    "ls200_horizon_tile": [_vp, _vp, _i, _i, _i, _i, _d, _f, _i, _i, _vp, _i64, _vp],
    "ls200_march_sites": [_vp, _vp, _i, _i, _i, _i, _i, _vp, _vp],
    "ls200_dem_set_heights_device": [_vp, _vp],
    "ls200_dem_level0_device": [_vp, _vp],
    "ls200_sun_loss_forward": [_vp, _vp, _i, _i, _i, _vp, _vp, _d, _vp, _vp],
    "ls200_sun_loss_backward": [_vp, _d, _vp, _i, _vp],
    "ls200_sun_loss_checkpoints": [_vp, _vp, _vp, _vp, _vp],
    "ls200_sun_loss_replay": [_vp, _vp],
    "ls200_capture_begin": [_vp],
    "ls200_capture_end": [_vp, _vp],
    "ls200_graph_launch": [_vp],
    "ls200_graph_nodes": [_vp, _vp],
    "ls200_graph_destroy": [_vp],
    "ls200_mission_duration_device": [_vp, _i, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _f, _f, _vp,
                                      _vp, _i, _i, _vp],
    "ls200_safe_haven_device": [_vp, _i, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _f, _f, _f, _vp,
                                _i, _vp],
    "ls200_earth_visibility_device": [_vp, _i, _vp, _vp, _vp, _vp, _vp, _vp, _f, _vp],
    "ls200_set_batch_config": [_vp, _i, _i],
    "ls200_get_batch_config": [_vp, _vp, _vp],
    "ls200_cbin_encode": [_vp, _f32p, _vp, _i64, _vp],
    "ls200_cbin_encode_device": [_vp, _vp, _vp, _vp],
    "ls200_cbin_decode": [_vp, _vp, _i64, _f32p],
    "ls200_vectors_create": [_vp, _f32p, _i, _vp],
    "ls200_vectors_destroy": [_vp],
    "ls200_lighting_load": [_vp, _f32p, _f64p, _f64p, _f32p, _i, _i, _i, _i],
    "ls200_lighting_run": [_vp, _vp, _i, _i, _i, _vp],
    "ls200_psr_run": [_vp, _vp, _vp],
    "ls200_psr_reduce_vectors": [_vp, _f32p, _i, _i, _f64p, _f64p, _f64p, _i, _vp, _vp],
    "ls200_memory_stats": [_i, _vp, _vp, _i],
    "ls200_lighting_device": [_vp, _i, _vp, _vp, _vp, _vp, _vp, _vp, _i, _i, _i, _vp, _vp],
    "ls200_sun_fraction": [_vp, _f32p, _f32p, _f32p, _i, _f32p],
    "ls200_lighting_device_noalloc": [_vp, _i, _vp, _vp, _vp, _vp, _vp, _vp, _i, _i, _i, _i,
                                      _vp],
    "ls200_host_alloc": [_i64, _vp],
    "ls200_host_free": [_vp],
    "ls200_fp32_probe": [_vp, _i, _vp],
    "ls200_check_arithmetic": [_vp, _vp, _vp],
}
_RESTYPES = {"ls200_last_error": ctypes.c_char_p, "ls200_abi_version": ctypes.c_int}


def register(name: str, argtypes: list, restype=ctypes.c_int) -> None:
    """Add a signature (used by modules that bind further entry points)."""
    SIGNATURES[name] = argtypes
    if restype is not ctypes.c_int:
        _RESTYPES[name] = restype
    if _lib is not None:
        function = getattr(_lib, name)
        function.argtypes = argtypes
        function.restype = restype


def library() -> ctypes.CDLL:
    """Load ``libls200.so`` once; raise CudaBackendError if it is missing."""
    global _lib
    with _lock:
        if _lib is None:
            if not LIBRARY_PATH.exists():
                raise CudaBackendError(
                    f"{LIBRARY_PATH.name} is not built; run __graft_entry__.build() "
                    "(nvcc for sm_100a) first"
                )
            try:
                loaded = ctypes.CDLL(str(LIBRARY_PATH))
            except OSError as error:
                raise CudaBackendError(f"cannot load {LIBRARY_PATH}: {error}") from error
            for name, argtypes in SIGNATURES.items():
                function = getattr(loaded, name)
                function.argtypes = argtypes
                function.restype = _RESTYPES.get(name, ctypes.c_int)
            _lib = loaded
        return _lib


def last_error() -> str:
    message = library().ls200_last_error()
    return message.decode(errors="replace") if message else ""


def check(status: int, what: str = "") -> None:
    """Map an ls200_status to the Python exception the reference raises."""
    if status == LS200_OK:
        return
    message = last_error()
    if what:
        message = f"{what}: {message}"
    if status == LS200_ERR_INVALID:
        raise ValueError(message)
    if status == LS200_ERR_UNAVAILABLE:
        raise CudaBackendError(message)
    if status == LS200_ERR_TIMEOUT:
        raise CudaTimeoutError(message)
    raise CudaExecutionError(message)


def call(name: str, *args) -> None:
    check(getattr(library(), name)(*args), name)


def exported_symbols() -> list[str]:
    return sorted(SIGNATURES)


def pinned_empty(shape, dtype=np.float32) -> np.ndarray:
    """Page-locked host array (cudaHostAlloc); freed when the last view dies."""
    dtype = np.dtype(dtype)
    shape = tuple(int(s) for s in np.atleast_1d(shape)) if not isinstance(shape, int) else (shape,)
    count = int(np.prod(shape, dtype=np.int64))
    nbytes = max(count * dtype.itemsize, 1)
    pointer = ctypes.c_void_p()
    call("ls200_host_alloc", nbytes, ctypes.byref(pointer))
    buffer = (ctypes.c_byte * nbytes).from_address(pointer.value)
    weakref.finalize(buffer, _free_host, pointer.value)
    return np.frombuffer(buffer, dtype=dtype, count=count).reshape(shape)


class PinnedPool:
    """Page-locked host arrays that recycle their memory.

    ``empty`` returns an ordinary writeable numpy array backed by pinned
    memory.  When its last view dies the buffer returns to the pool (at most
    ``keep`` idle buffers per size; others are freed), so a caller that drops
    each result before the next call gets device-to-host copies at full DMA
    speed into memory that is already mapped, instead of a fresh pageable
    array faulted in page by page."""

    def __init__(self, keep: int = 2) -> None:
        self._idle: dict[int, list[int]] = {}
        self._keep = keep
        self._lock = threading.Lock()

    def empty(self, shape, dtype=np.float32) -> np.ndarray:
        dtype = np.dtype(dtype)
        shape = tuple(int(s) for s in shape) if not isinstance(shape, int) else (shape,)
        count = int(np.prod(shape, dtype=np.int64))
        nbytes = max(count * dtype.itemsize, 1)
        with self._lock:
            stack = self._idle.get(nbytes)
            address = stack.pop() if stack else None
        if address is None:
            pointer = ctypes.c_void_p()
            call("ls200_host_alloc", nbytes, ctypes.byref(pointer))
            address = pointer.value
        buffer = (ctypes.c_byte * nbytes).from_address(address)
        weakref.finalize(buffer, self._release, address, nbytes)
        return np.frombuffer(buffer, dtype=dtype, count=count).reshape(shape)

    def _release(self, address: int, nbytes: int) -> None:
        with self._lock:
            stack = self._idle.setdefault(nbytes, [])
            if len(stack) < self._keep:
                stack.append(address)
                return
        _free_host(address)


def _free_host(address: int) -> None:
    try:
        library().ls200_host_free(ctypes.c_void_p(address))
    except Exception:  # pragma: no cover - interpreter shutdown
        pass


def memory_stats(device: int = 0, *, reset_peak: bool = False) -> tuple[int, int]:
    """(bytes in use, high-water mark) of this library's own device
    allocations on `device` (ls200_memory_stats)."""
    in_use, peak = ctypes.c_int64(0), ctypes.c_int64(0)
    call("ls200_memory_stats", int(device), ctypes.byref(in_use), ctypes.byref(peak),
         1 if reset_peak else 0)
    return int(in_use.value), int(peak.value)
