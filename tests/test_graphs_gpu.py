"""CUDA-graph-captured lighting time chunks on the B200: a recorded sequence
of chunked ls200_lighting_device calls replays to the eager results, also
after the input buffers are refilled."""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

from test_oracle_lighting_pins import synthetic_horizons

pytestmark = pytest.mark.gpu

TILES = 2
BLOCK = 1024


@pytest.fixture(scope="module")
def lighting_inputs(cuda_session):
    import torch

    from lunarscout_b200 import synthetic
    from lunarscout_b200.contract import projection_array
    from lunarscout_b200.lightmap_cuda import DeviceVectors

    dem = synthetic.config1_dem()
    horizons = torch.from_numpy(np.stack([synthetic_horizons(), synthetic_horizons() + 1.5])
                                .reshape(TILES, 128 * 128, 1440)).cuda()
    patches = torch.from_numpy(np.stack([dem.elevation_m[128:256, 128:256],
                                         dem.elevation_m[256:384, 128:256]])).cuda()
    geo = np.ascontiguousarray(np.repeat(dem.geo_transform[None], TILES, 0))
    proj = np.ascontiguousarray(np.repeat(projection_array(dem.projection)[None], TILES, 0))
    windows = np.array([[128, 128, 128, 128], [128, 256, 128, 100]], dtype=np.int32)
    hours = synthetic.hours_between("2030-01-01T00", "2030-05-01T00", 1.0)[:2600]
    table = DeviceVectors(cuda_session.context, synthetic.sun_vectors(hours).astype(np.float32))
    frames = torch.empty(TILES * 128 * 128 * 12, dtype=torch.float32, device="cuda")
    blocks = [(start, min(BLOCK, len(hours) - start)) for start in range(0, len(hours), BLOCK)]
    yield dict(horizons=horizons, patches=patches, geo=geo, proj=proj, windows=windows,
               table=table, frames=frames, blocks=blocks)
    table.close()


def _chunks(session, inputs, outs):
    from lunarscout_b200 import _native

    lib = _native.library()
    for (start, count), out in zip(inputs["blocks"], outs):
        _native.check(lib.ls200_lighting_device(
            session.context, TILES, ctypes.c_void_p(inputs["patches"].data_ptr()),
            inputs["geo"].ctypes.data, inputs["proj"].ctypes.data, inputs["windows"].ctypes.data,
            ctypes.c_void_p(inputs["horizons"].data_ptr()), inputs["table"].handle, start, count,
            1, ctypes.c_void_p(inputs["frames"].data_ptr()), ctypes.c_void_p(out.data_ptr())))


def _outputs(inputs):
    import torch

    return [torch.zeros((TILES, count, 128 * 128), dtype=torch.uint8, device="cuda")
            for _, count in inputs["blocks"]]


def test_replayed_chunks_equal_the_eager_launches(cuda_session, lighting_inputs):
    import torch

    from lunarscout_b200.graphs import DeviceGraph

    eager = _outputs(lighting_inputs)
    torch.cuda.synchronize()
    _chunks(cuda_session, lighting_inputs, eager)
    cuda_session.synchronize()
    replayed = _outputs(lighting_inputs)
    torch.cuda.synchronize()
    with DeviceGraph.capture(cuda_session.context,
                             lambda: _chunks(cuda_session, lighting_inputs, replayed)) as graph:
        cuda_session.synchronize()
        assert all(int(o.sum()) == 0 for o in replayed)  # recorded, not run
        assert graph.nodes >= 2 * len(lighting_inputs["blocks"])
        graph.launch()
        cuda_session.synchronize()
        for a, b in zip(eager, replayed):
            assert torch.equal(a, b)
        assert sum(int(o.float().mean() > 0) for o in eager) > 0
        # Refill the inputs the graph reads and replay: the next "tile".
        lighting_inputs["horizons"].add_(-3.0)
        torch.cuda.synchronize()
        graph.launch()
        cuda_session.synchronize()
        _chunks(cuda_session, lighting_inputs, eager)
        cuda_session.synchronize()
        for a, b in zip(eager, replayed):
            assert torch.equal(a, b)
        lighting_inputs["horizons"].add_(3.0)
        torch.cuda.synchronize()


def test_capture_needs_a_created_stream(cuda_session):
    from lunarscout_b200.graphs import DeviceGraph

    cuda_session.set_stream(0)
    try:
        with pytest.raises(ValueError):
            DeviceGraph.capture(cuda_session.context, lambda: None)
    finally:
        cuda_session.set_stream(None)


def test_ordered_sub_ranges_equal_the_whole_launch_and_time_order(cuda_session,
                                                                     lighting_inputs):
    """Chunks of the time axis (each visiting its steps in longitude order
    through the compacted order window) equal one whole-axis launch, which
    equals time-order evaluation (the per-patch session, 32 steps a call)."""
    import torch

    from lunarscout_b200 import _native, synthetic
    from lunarscout_b200.lightmap_cuda import LightmapCudaSession

    inputs = lighting_inputs
    outs = _outputs(inputs)
    _chunks(cuda_session, inputs, outs)
    total = sum(count for _, count in inputs["blocks"])
    whole = torch.zeros((TILES, total, 128 * 128), dtype=torch.uint8, device="cuda")
    _native.check(_native.library().ls200_lighting_device(
        cuda_session.context, TILES, ctypes.c_void_p(inputs["patches"].data_ptr()),
        inputs["geo"].ctypes.data, inputs["proj"].ctypes.data, inputs["windows"].ctypes.data,
        ctypes.c_void_p(inputs["horizons"].data_ptr()), inputs["table"].handle, 0, total, 1,
        ctypes.c_void_p(inputs["frames"].data_ptr()), ctypes.c_void_p(whole.data_ptr())))
    cuda_session.synchronize()
    torch.cuda.synchronize()
    np.testing.assert_array_equal(torch.cat(outs, dim=1).cpu().numpy(), whole.cpu().numpy())
    dem = synthetic.config1_dem()
    hours = synthetic.hours_between("2030-01-01T00", "2030-05-01T00", 1.0)[:total]
    session = LightmapCudaSession(time_batch_size=32)
    try:
        tile_x, tile_y, vw, vh = (int(v) for v in inputs["windows"][1])
        horizons = inputs["horizons"][1].view(128, 128, 1440).cpu().numpy()
        expected = np.stack(list(session.iter_patch_tiles(
            dem, horizons, synthetic.sun_vectors(hours), tile_y=tile_y, tile_x=tile_x,
            valid_height=vh, valid_width=vw)))
    finally:
        session.close()
    got = whole[1].cpu().numpy().reshape(total, 128, 128)[:, :vh, :vw]
    np.testing.assert_array_equal(got, expected)
