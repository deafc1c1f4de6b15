"""ORACLE — test infrastructure only.

CPU restatements of lunarscout's horizon-and-lighting hot path, used to check
the CUDA implementation in ``lunarscout_b200``.  Only ``tests/``,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` import this
package; the product path never does.

* ``march_oracle.c`` restates the production horizon march
  (src/lunarscout/_numba_horizon/cuda_backend.py:656-874, :965-1134) in FP32
  with every rounding written out, plus an FP64 twin, and the factor-four max
  pyramid (src/lunarscout/_numba_horizon/pyramid.py:19-138).
* ``segments.c`` restates host segment generation
  (src/lunarscout/_numba_horizon/geometry_numba.py:30-364 and
  geometry.py:255-487, 575-673).
* ``lighting.c`` restates the lightmap / margin / PSR per-pixel arithmetic
  (src/lunarscout/_numba_horizon/lightmap_cpu.py:25-183, psr.py:29-140).
* ``products.py`` restates the PSR vector reduction, the mission-duration
  reducer and the ``.cbin`` codec in NumPy.

Parity pins: the golden captures of the reference (C# production kernel
outputs shipped in the reference's tests/data/numba_horizon) and fixtures
generated by importing the reference's own Python in this container
(tests/golden/make_golden.py).
"""

from __future__ import annotations

import ctypes
import os
import subprocess
import threading
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
_LIB = None
_LIB_LOCK = threading.Lock()

# FMA contraction groups (march_oracle.c ORA_CF_*).
CF_EVAL = 1 << 0
CF_TAN = 1 << 1
CF_PLANAR = 1 << 2
CF_CHORD = 1 << 3
CF_TRUEM = 1 << 4
CF_NEAR = 1 << 5
CF_BOUND = 1 << 6
CF_SLOPE = 1 << 7
CF_MAG = 1 << 8
CF_BILIN = 1 << 9
CF_RES = 1 << 10
CF_ALL = (1 << 11) - 1
CF_PLANAR_ALT = 1 << 11
CF_CHORD_ALT = 1 << 12
CF_MAG_ALT = 1 << 13
CF_SLOPE_ALT = 1 << 14
CF_BOUND_ALT = 1 << 15
CF_RES_ALT = 1 << 17
CF_LXS_ALT = 1 << 18
CF_SHIFT = 1 << 19
#: Superseded level-0 cell-exit step cap (only to pin the older golden capture).
OPT_EXIT_CAP = 1 << 16
#: Skip ladder of the batched traversal (no reference counterpart): a cull
#: climbs to the largest culled ancestor cell before skipping.
OPT_LADDER = 1 << 20
#: Relative-height level-0 slopes (this project's accuracy mode): local z from
#: height - observer_z and 2R + height + observer_z, never from R + height
#: rounded on its own.
OPT_RELATIVE = 1 << 21


def ladder_mask(cap: int = 0, min_km: int = 0, base: int | None = None) -> int:
    """Production arithmetic with the skip ladder; ``cap`` limits the climb
    (0 = up to the top level), ``min_km`` is the distance from which it acts."""
    if not 0 <= cap <= 15 or not 0 <= min_km <= 15:
        raise ValueError("ladder cap and distance must be between 0 and 15")
    return (PRODUCTION_MASK if base is None else base) | OPT_LADDER | (cap << 24) | (min_km << 28)

#: Contraction mask whose FP32 arithmetic reproduces the golden captures of
#: the reference's C# production kernel (tests/test_oracle_pins.py checks it):
#: local_x^2 = dist * dist - local_z^2 fuses dist * dist.
CSHARP_MASK = (
    CF_EVAL | CF_TAN | CF_PLANAR | CF_CHORD | CF_CHORD_ALT | CF_TRUEM | CF_NEAR
    | CF_BOUND | CF_SLOPE | CF_MAG | CF_BILIN | CF_RES | CF_LXS_ALT | CF_SHIFT
)
#: The reference's runtime arithmetic: its Numba-CUDA kernel
#: (cuda_backend.py:656-1134) as NVVM compiles it, run on a B200; the same as
#: the C# captures except that local_x^2 fuses local_z * local_z (pinned by
#: tests/golden/numba_cuda_b200.npz).  The product marches with it.
PRODUCTION_MASK = CSHARP_MASK & ~CF_LXS_ALT


def build(force: bool = False) -> Path:
    """Compile ``liboracle.so`` in place with the committed Makefile."""
    target = HERE / "liboracle.so"
    if force or not target.exists() or _stale(target):
        subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return target


def _stale(target: Path) -> bool:
    built = target.stat().st_mtime
    return any(
        path.stat().st_mtime > built
        for pattern in ("*.c", "*.inc", "*.h", "Makefile")
        for path in HERE.glob(pattern)
    )


def lib() -> ctypes.CDLL:
    global _LIB
    with _LIB_LOCK:
        if _LIB is None:
            path = HERE / "liboracle.so"
            if not path.exists():
                build()
            _LIB = ctypes.CDLL(str(path))
            _declare(_LIB)
        return _LIB


_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")
_c = ctypes


def _declare(library: ctypes.CDLL) -> None:
    march_args = [
        _f32p, _c.c_int, _c.c_int, _c.c_int,
        _f32p, _c.c_int, _c.c_int, _f32p,
        _f32p, _c.c_int, _c.c_int, _f32p, _i32p, _c.c_int, _f32p, _f32p,
        _c.c_int, _c.c_int, _c.c_int, _c.c_int, _c.c_int, _c.c_int, _c.c_float,
        _c.c_void_p, _c.c_void_p, _c.c_longlong,
    ]
    library.ora_march_pass_f32.argtypes = march_args + [_f32p, _c.c_uint, _c.c_int, _i64p]
    library.ora_march_pass_f32.restype = _c.c_int
    library.ora_march_pass_f64.argtypes = march_args + [_f64p, _c.c_uint, _c.c_int, _i64p]
    library.ora_march_pass_f64.restype = _c.c_int
    library.ora_march_trace_f32.argtypes = march_args + [_f32p, _c.c_uint, _f32p, _c.c_int]
    library.ora_march_trace_f32.restype = _c.c_int
    library.ora_march_trace_f64.argtypes = march_args + [_f64p, _c.c_uint, _f32p, _c.c_int]
    library.ora_march_trace_f64.restype = _c.c_int
    library.ora_hierarchy_maximum_f32.argtypes = [
        _f32p, _f32p, _c.c_int, _c.c_int, _f32p, _i32p, _c.c_int,
        _c.c_float, _c.c_float, _c.c_float, _c.c_int, _c.c_float, _c.c_uint,
        _c.c_void_p, _c.c_int, _c.c_void_p,
    ]
    library.ora_hierarchy_maximum_f32.restype = _c.c_float
    library.ora_pyramid_layout.argtypes = [_c.c_int, _c.c_int, _c.c_void_p, _c.c_void_p]
    library.ora_pyramid_layout.restype = _c.c_int
    library.ora_build_pyramid.argtypes = [_f32p, _c.c_int, _c.c_int, _f32p]
    library.ora_build_pyramid.restype = _c.c_int
    for name, argtypes, restype in _EXTRA_DECLARATIONS:
        if hasattr(library, name):
            function = getattr(library, name)
            function.argtypes = argtypes
            function.restype = restype


_EXTRA_DECLARATIONS: list = []


def _declare_extra(name: str, argtypes: list, restype) -> None:
    """Register a ctypes signature from a submodule (applied on load)."""
    _EXTRA_DECLARATIONS.append((name, argtypes, restype))
    if _LIB is not None and hasattr(_LIB, name):
        function = getattr(_LIB, name)
        function.argtypes = argtypes
        function.restype = restype


def default_threads() -> int:
    return max(1, len(os.sched_getaffinity(0)))


# --------------------------------------------------------------------------
# pyramid
# --------------------------------------------------------------------------

def pyramid_layout(width: int, height: int) -> tuple[np.ndarray, int]:
    library = lib()
    count = library.ora_pyramid_layout(int(width), int(height), None, None)
    levels = np.zeros((count, 4), dtype=np.int32)
    mip_count = ctypes.c_longlong(0)
    library.ora_pyramid_layout(
        int(width), int(height), levels.ctypes.data, ctypes.addressof(mip_count)
    )
    return levels, int(mip_count.value)


def build_pyramid(level0: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """Return (mips, levels) of the factor-four valid-max pyramid."""
    level0 = np.ascontiguousarray(level0, dtype=np.float32)
    height, width = level0.shape
    levels, mip_count = pyramid_layout(width, height)
    mips = np.empty(max(mip_count, 1), dtype=np.float32)
    lib().ora_build_pyramid(level0, width, height, mips)
    return mips[:mip_count].copy(), levels


# --------------------------------------------------------------------------
# horizon march
# --------------------------------------------------------------------------

def _pyr_args(pyramid) -> list:
    level0 = np.ascontiguousarray(pyramid.level0, dtype=np.float32)
    mips = np.ascontiguousarray(pyramid.mips, dtype=np.float32)
    if mips.size == 0:
        mips = np.zeros(1, dtype=np.float32)
    return [
        level0, level0.shape[1], level0.shape[0], mips,
        np.ascontiguousarray(pyramid.levels, dtype=np.int32), len(pyramid.levels),
        np.ascontiguousarray(pyramid.map_parameters, dtype=np.float32),
        np.ascontiguousarray(pyramid.projection_parameters, dtype=np.float32),
    ]


def march_pass(
    segments: np.ndarray,
    primary,
    active,
    *,
    tile_column: int,
    tile_row: int,
    tile_width: int,
    tile_height: int,
    subpatch_size: int,
    pass_index: int,
    observer_elevation_m: float = 0.0,
    slopes: np.ndarray | None = None,
    pixels: np.ndarray | None = None,
    azimuths: np.ndarray | None = None,
    precision: str = "f32",
    mask: int = PRODUCTION_MASK,
    threads: int | None = None,
) -> tuple[np.ndarray, tuple[int, int]]:
    """One DEM pass of the production march.

    Full tile: returns slopes ``[tile_width*tile_height, A]`` (pixel-major).
    With ``pixels``/``azimuths`` lists: returns one slope per listed ray.
    Also returns (node visits, level-0 samples).
    """
    segments = np.ascontiguousarray(segments, dtype=np.float32)
    azimuth_count, center_count, dem_count, fields = segments.shape
    if fields != 18:
        raise ValueError("segments must be [A, C, D, 18]")
    dtype = np.float32 if precision == "f32" else np.float64
    if pixels is not None:
        pixels = np.ascontiguousarray(pixels, dtype=np.int32)
        azimuths = np.ascontiguousarray(azimuths, dtype=np.int32)
        shape = pixels.shape
    else:
        shape = (tile_width * tile_height, azimuth_count)
    if slopes is None:
        out = np.full(shape, -np.inf, dtype=dtype)
    else:
        out = np.array(slopes, dtype=dtype, copy=True).reshape(shape)
    primary_level0 = np.ascontiguousarray(primary.level0, dtype=np.float32)
    counters = np.zeros(2, dtype=np.int64)
    args = [
        segments, azimuth_count, center_count, dem_count,
        primary_level0, primary_level0.shape[1], primary_level0.shape[0],
        np.ascontiguousarray(primary.map_parameters, dtype=np.float32),
        *_pyr_args(active),
        tile_column, tile_row, tile_width, tile_height, subpatch_size, pass_index,
        float(observer_elevation_m),
        None if pixels is None else pixels.ctypes.data,
        None if pixels is None else azimuths.ctypes.data,
        0 if pixels is None else pixels.size,
    ]
    function = lib().ora_march_pass_f32 if precision == "f32" else lib().ora_march_pass_f64
    function(*args, out, int(mask), int(threads or default_threads()), counters)
    return out, (int(counters[0]), int(counters[1]))


def march_all_passes(
    segments: np.ndarray,
    pyramids,
    *,
    tile_column: int,
    tile_row: int,
    tile_width: int = 128,
    tile_height: int = 128,
    subpatch_size: int = 8,
    observer_elevation_m: float = 0.0,
    pixels: np.ndarray | None = None,
    azimuths: np.ndarray | None = None,
    precision: str = "f32",
    mask: int = PRODUCTION_MASK,
    threads: int | None = None,
) -> tuple[np.ndarray, tuple[int, int]]:
    """Every DEM pass on one carried slope buffer (cuda_backend.py:1445-1552)."""
    slopes = None
    visits = samples = 0
    for pass_index, active in enumerate(pyramids):
        slopes, (v, s) = march_pass(
            segments, pyramids[0], active, tile_column=tile_column, tile_row=tile_row,
            tile_width=tile_width, tile_height=tile_height, subpatch_size=subpatch_size,
            pass_index=pass_index, observer_elevation_m=observer_elevation_m,
            slopes=slopes, pixels=pixels, azimuths=azimuths, precision=precision,
            mask=mask, threads=threads,
        )
        visits += v
        samples += s
    return slopes, (visits, samples)


def march_trace(
    segments, primary, active, *, tile_column, tile_row, tile_width, tile_height,
    subpatch_size, pass_index, pixel, azimuth, observer_elevation_m=0.0,
    initial=-np.inf, mask=PRODUCTION_MASK, capacity=65536, precision="f32",
) -> tuple[float, np.ndarray]:
    """One ray of one pass with its 12-field branch trace (rows in float32)."""
    segments = np.ascontiguousarray(segments, dtype=np.float32)
    azimuth_count, center_count, dem_count, _ = segments.shape
    primary_level0 = np.ascontiguousarray(primary.level0, dtype=np.float32)
    slope = np.array([initial], dtype=np.float32 if precision == "f32" else np.float64)
    function = lib().ora_march_trace_f32 if precision == "f32" else lib().ora_march_trace_f64
    rows = np.zeros((capacity, 12), dtype=np.float32)
    pixels = np.array([pixel], dtype=np.int32)
    azimuths = np.array([azimuth], dtype=np.int32)
    count = function(
        segments, azimuth_count, center_count, dem_count,
        primary_level0, primary_level0.shape[1], primary_level0.shape[0],
        np.ascontiguousarray(primary.map_parameters, dtype=np.float32),
        *_pyr_args(active),
        tile_column, tile_row, tile_width, tile_height, subpatch_size, pass_index,
        float(observer_elevation_m), pixels.ctypes.data, azimuths.ctypes.data, 1,
        slope, int(mask), rows, capacity,
    )
    return float(slope[0]), rows[:count].copy()


def hierarchy_maximum(
    segment16, pyramid, *, observer_z, radius, resolution, pass_index,
    initial=-np.inf, mask=PRODUCTION_MASK, capacity=0,
):
    """The bare march of one interpolated segment (fields 0,1,4..17)."""
    level0 = np.ascontiguousarray(pyramid.level0, dtype=np.float32)
    mips = np.ascontiguousarray(pyramid.mips, dtype=np.float32)
    if mips.size == 0:
        mips = np.zeros(1, dtype=np.float32)
    rows = np.zeros((max(capacity, 1), 12), dtype=np.float32)
    count = ctypes.c_int(0)
    value = lib().ora_hierarchy_maximum_f32(
        np.ascontiguousarray(segment16, dtype=np.float32), level0, level0.shape[1],
        level0.shape[0], mips, np.ascontiguousarray(pyramid.levels, dtype=np.int32),
        len(pyramid.levels), observer_z, radius, resolution, pass_index, initial,
        int(mask), rows.ctypes.data if capacity else None, capacity,
        ctypes.addressof(count),
    )
    return float(value), rows[: count.value].copy()


SEGMENT_MARCH_FIELDS = (0, 1, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15, 16, 17)
