"""The allocation-free lighting entry point against the allocating one.

ls200_lighting_device_noalloc serves callers that may not call cudaMalloc
while they run (their device memory is owned by another allocator, or an
allocation's device-wide synchronisation is not affordable).  It keeps its
frame scratch in a fixed device array inside the library instead of taking
it from the caller.  Its results must equal ls200_lighting_device's on the
same inputs, call after call, because both run the same kernels; it must also
refuse batches larger than its scratch.

This file is collected last on purpose, and builds everything it needs
itself, so it passes alone in a fresh process and after the other tests.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TILES = 3
PLANE = 128 * 128


def _horizons(seed):
    az = np.radians(np.arange(1440, dtype=np.float64) * 0.25)
    y, x = np.mgrid[0:128, 0:128]
    phase = (0.05 * x + 0.03 * y + seed)[..., None]
    level = (1.0 + 0.1 * (x - y) + seed)[..., None]
    h = level + 2.5 * np.sin(3.0 * az + phase) + np.sin(11.0 * az + 2.0 * phase)
    return np.ascontiguousarray(h, dtype=np.float32)


@pytest.fixture(scope="module")
def inputs():
    import torch

    from lunarscout_b200 import synthetic
    from lunarscout_b200.contract import projection_array

    dem = synthetic.config1_dem()
    hours = synthetic.hours_between("2029-01-01T00", "2029-02-01T00", 6.0)
    vectors = synthetic.sun_vectors(hours).astype(np.float32)
    windows = np.array([[0, 0, 128, 128], [256, 128, 128, 128], [448, 448, 64, 64]],
                       dtype=np.int32)[:TILES]
    patches = np.zeros((TILES, 128, 128), dtype=np.float32)
    for t, (tx, ty, vw, vh) in enumerate(windows):
        patches[t, :vh, :vw] = dem.elevation_m[ty:ty + vh, tx:tx + vw]
    horizons = np.stack([_horizons(0.3 * t) for t in range(TILES)])
    geo = np.ascontiguousarray(np.repeat(dem.geo_transform[None, :], TILES, 0))
    proj = np.ascontiguousarray(np.repeat(projection_array(dem.projection)[None, :], TILES, 0))
    device = torch.device("cuda", 0)
    return dict(
        patches=torch.from_numpy(patches).to(device),
        horizons=torch.from_numpy(horizons).to(device),
        vectors=torch.from_numpy(vectors).to(device),
        host_vectors=vectors, windows=windows, geo=geo, proj=proj,
    )


def test_no_alloc_entry_point_matches_the_allocating_one_on_consecutive_calls(inputs):
    import torch

    from lunarscout_b200 import _native
    from lunarscout_b200.lightmap_cuda import DeviceVectors, LightingContext

    lib = _native.library()
    context = LightingContext(0)
    try:
        stream = torch.cuda.current_stream()
        _native.call("ls200_set_stream", context.handle, ctypes.c_void_p(stream.cuda_stream))
        table = DeviceVectors(context.handle, inputs["host_vectors"])
        count = len(inputs["host_vectors"])
        frames = torch.empty(TILES * PLANE * 12, dtype=torch.float32, device="cuda")
        # (time start, time count, signal, output type); signal 3 (PSR) runs
        # over the whole table and writes one plane per tile.
        calls = [(0, 40, 0, torch.float32), (40, count - 40, 1, torch.uint8),
                 (5, 64, 2, torch.float32), (0, count, 3, torch.uint8)]
        for start, length, signal, dtype in calls:
            shape = (TILES, PLANE) if signal == 3 else (TILES, length, PLANE)
            expected = torch.full(shape, 7, dtype=dtype, device="cuda")
            got = torch.full(shape, 9, dtype=dtype, device="cuda")
            torch.cuda.synchronize()
            _native.check(lib.ls200_lighting_device(
                context.handle, TILES, ctypes.c_void_p(inputs["patches"].data_ptr()),
                inputs["geo"].ctypes.data, inputs["proj"].ctypes.data,
                inputs["windows"].ctypes.data, ctypes.c_void_p(inputs["horizons"].data_ptr()),
                table.handle, start, length, signal, ctypes.c_void_p(frames.data_ptr()),
                ctypes.c_void_p(expected.data_ptr())))
            _native.check(lib.ls200_lighting_device_noalloc(
                context.handle, TILES, ctypes.c_void_p(inputs["patches"].data_ptr()),
                inputs["geo"].ctypes.data, inputs["proj"].ctypes.data,
                inputs["windows"].ctypes.data, ctypes.c_void_p(inputs["horizons"].data_ptr()),
                ctypes.c_void_p(inputs["vectors"].data_ptr()), count, start, length, signal,
                ctypes.c_void_p(got.data_ptr())))
            torch.cuda.synchronize()
            # Same kernels on the same inputs: equal, well inside the 1e-4
            # fraction tolerance of the lighting tests.
            assert torch.equal(got, expected), (start, length, signal)
        table.close()
    finally:
        context.close()


def test_no_alloc_entry_point_takes_no_device_memory(inputs):
    """After a first call on the device (which loads the kernels and looks up
    the scratch address), further calls leave the device's free memory as it
    was."""
    import torch

    from lunarscout_b200 import _native
    from lunarscout_b200.lightmap_cuda import LightingContext

    lib = _native.library()
    context = LightingContext(0)
    try:
        stream = torch.cuda.current_stream()
        _native.call("ls200_set_stream", context.handle, ctypes.c_void_p(stream.cuda_stream))
        count = len(inputs["host_vectors"])
        out = torch.empty((TILES, count, PLANE), dtype=torch.uint8, device="cuda")

        def run():
            _native.check(lib.ls200_lighting_device_noalloc(
                context.handle, TILES, ctypes.c_void_p(inputs["patches"].data_ptr()),
                inputs["geo"].ctypes.data, inputs["proj"].ctypes.data,
                inputs["windows"].ctypes.data, ctypes.c_void_p(inputs["horizons"].data_ptr()),
                ctypes.c_void_p(inputs["vectors"].data_ptr()), count, 0, count, 1,
                ctypes.c_void_p(out.data_ptr())))
            torch.cuda.synchronize()

        run()
        free_before, _ = torch.cuda.mem_get_info(0)
        run()
        run()
        free_after, _ = torch.cuda.mem_get_info(0)
        assert free_after == free_before
    finally:
        context.close()


def test_no_alloc_entry_point_rejects_batches_beyond_its_scratch(inputs):
    from lunarscout_b200 import _native
    from lunarscout_b200.lightmap_cuda import LightingContext

    lib = _native.library()
    context = LightingContext(0)
    try:
        five = np.zeros((5, 4), dtype=np.int32)
        geo = np.zeros((5, 6))
        status = lib.ls200_lighting_device_noalloc(
            context.handle, 5, ctypes.c_void_p(inputs["patches"].data_ptr()),
            geo.ctypes.data, geo.ctypes.data, five.ctypes.data,
            ctypes.c_void_p(inputs["horizons"].data_ptr()),
            ctypes.c_void_p(inputs["vectors"].data_ptr()), 10, 0, 10, 0,
            ctypes.c_void_p(inputs["horizons"].data_ptr()))
        assert status == _native.LS200_ERR_INVALID
        assert "1 to 4 tiles" in _native.last_error()
    finally:
        context.close()
