"""Horizon tiles on the B200: the .cbin codec against the reference encoder's
golden payload, and ``ls200_horizon_tile`` (segments -> passes -> degrees ->
codec on the device) against the step-by-step device path and the oracle."""

from __future__ import annotations

import ctypes
import hashlib

import numpy as np
import pytest

import oracle
from oracle import products
from oracle import segments as oseg
from conftest import load_golden
from test_oracle_lighting_pins import synthetic_horizons

pytestmark = pytest.mark.gpu

AZ = 1440


def _codec_input() -> np.ndarray:
    degrees = synthetic_horizons().reshape(-1, AZ) * np.float32(6.0)
    degrees[5, :7] = -np.inf
    degrees[9, 100:110] = 75.0
    return np.ascontiguousarray(degrees, dtype=np.float32)


@pytest.fixture(scope="module")
def codec(cuda_session):
    from lunarscout_b200.file_format import TileCodec

    return TileCodec(context=cuda_session.context)


@pytest.fixture(scope="module")
def synthetic_pair():
    from lunarscout_b200.synthetic import SyntheticDemSpec, synthetic_dem

    primary = synthetic_dem(SyntheticDemSpec(320, 20.0, craters=30, seed=5))
    regional = synthetic_dem(SyntheticDemSpec(400, 240.0, sigma_m=1200.0, craters=0,
                                              tilt_m=2000.0, seed=1005))
    return primary, regional


def _tile(session, dems, *, tile_x, tile_y, azimuths, distance, observer, compress=False):
    handles = (ctypes.c_void_p * len(dems))(*[d.handle.value for d in dems])
    capacity = 16384 * (2 * AZ + 2) if compress else 16384 * azimuths * 4
    out = np.empty(capacity, dtype=np.uint8)
    size = ctypes.c_int64()
    from lunarscout_b200._native import call

    call("ls200_horizon_tile", session.context, handles, len(dems), tile_x, tile_y, azimuths,
         float(distance), float(observer), 8, 1 if compress else 0, out.ctypes.data, capacity,
         ctypes.byref(size))
    return out[: size.value]


def test_device_encoder_reproduces_the_reference_payload(codec):
    arrays = load_golden("codec_reference.npz")
    payload = codec.encode(_codec_input())
    assert len(payload) == int(arrays["payload_size"])
    assert hashlib.sha256(payload).hexdigest() == str(arrays["payload_sha256"])
    lengths = np.empty(16384, dtype=np.int64)
    offset = 0
    for pixel in range(16384):
        lengths[pixel] = payload[offset] | (payload[offset + 1] << 8)
        offset += 2 + int(lengths[pixel])
    np.testing.assert_array_equal(lengths, arrays["lengths"])


def test_device_decoder_matches_the_oracle_decoder(codec):
    arrays = load_golden("codec_reference.npz")
    payload = products.encode_tile(_codec_input())
    decoded = codec.decode(payload)
    np.testing.assert_array_equal(decoded[[0, 5, 9, 777, 16383]], arrays["decoded_rows"])
    np.testing.assert_array_equal(decoded[::97], products.decode_tile(payload)[::97])


def test_device_decoder_rejects_truncated_and_trailing_payloads(codec):
    payload = codec.encode(_codec_input())
    with pytest.raises(ValueError):
        codec.decode(payload[:-1])
    with pytest.raises(ValueError):
        codec.decode(payload + b"\x00")


def test_clamped_deltas_match_the_oracle_encoder(codec):
    # Jumps beyond +-16383 quanta (about 25 degrees) are clamped by the
    # format, so the first rows are compared block by block with the oracle.
    rng = np.random.default_rng(11)
    degrees = rng.uniform(-49.0, 49.0, size=(16384, AZ)).astype(np.float32)
    degrees[1] = np.where(np.arange(AZ) % 2 == 0, -49.0, 49.0)
    degrees[2] = 0.0
    degrees[3, ::5] = np.inf
    payload = codec.encode(degrees)
    head = products.encode_tile(degrees[:6])
    assert payload[: len(head)] == head
    decoded = codec.decode(payload)
    rows = np.frombuffer(payload, np.uint8)
    np.testing.assert_array_equal(decoded[:6], _oracle_rows(rows, 6))


def _oracle_rows(payload: np.ndarray, count: int) -> np.ndarray:
    offset = 0
    blocks = []
    for _ in range(count):
        length = int(payload[offset]) | (int(payload[offset + 1]) << 8)
        blocks.append(payload[offset: offset + 2 + length].tobytes())
        offset += 2 + length
    # decode_tile wants a whole tile: repeat the last block to 16384 pixels.
    whole = b"".join(blocks) + blocks[-1] * (16384 - count)
    return products.decode_tile(whole)[:count]


def test_smooth_tiles_round_trip_within_half_a_quantum(codec):
    rng = np.random.default_rng(12)
    walk = np.cumsum(rng.normal(0.0, 0.5, size=(16384, AZ)), axis=1)
    degrees = np.clip(walk, -49.0, 49.0).astype(np.float32)
    decoded = codec.decode(codec.encode(degrees))
    step = np.float32(50.0) / np.float32(32767.0)
    # half a quantum, plus the float32 rounding of scale-up and scale-down
    assert np.max(np.abs(decoded - degrees)) <= step * 0.51


def test_tile_entry_equals_the_step_by_step_device_path(synthetic_pair, cuda_session):
    primary, regional = synthetic_pair
    dems = [cuda_session.upload_dem_grid(primary), cuda_session.upload_dem_grid(regional)]
    tile = dict(tile_column=128, tile_row=128, tile_width=128, subpatch_size=8)
    raw = _tile(cuda_session, dems, tile_x=128, tile_y=128, azimuths=48, distance=150_000.0,
                observer=1.5)
    got = raw.view("<f4").reshape(16384, 48)
    segments = cuda_session.generate_segments(dems, azimuth_count=48,
                                              maximum_distance_m=150_000.0,
                                              observer_elevation_m=1.5, **tile)
    pyramids = [cuda_session.build_max_pyramid(primary), cuda_session.build_max_pyramid(regional)]
    slopes, _ = cuda_session.subpatch_hierarchical_all_passes(
        segments, pyramids, tile_height=128, observer_elevation_m=1.5, **tile)
    np.testing.assert_array_equal(got, cuda_session.slopes_to_degrees(slopes))


def test_tile_entry_agrees_with_the_oracle_within_a_hundredth_degree(synthetic_pair,
                                                                      cuda_session):
    from lunarscout_b200.contract import HorizonBuffers, PyramidArrays, map_parameters
    from lunarscout_b200.contract import projection_parameters

    primary, regional = synthetic_pair
    dems = [cuda_session.upload_dem_grid(primary), cuda_session.upload_dem_grid(regional)]
    raw = _tile(cuda_session, dems, tile_x=0, tile_y=128, azimuths=36, distance=150_000.0,
                observer=0.0)
    got = raw.view("<f4").reshape(16384, 36)
    tile = dict(tile_column=0, tile_row=128, tile_width=128, subpatch_size=8)
    segments = oseg.build_segments([primary, regional], azimuth_count=36,
                                   maximum_distance_m=150_000.0, **tile)
    pyramids = []
    for dem in (primary, regional):
        mips, levels = oracle.build_pyramid(dem.elevation_m)
        pyramids.append(PyramidArrays(dem.elevation_m, mips, levels, map_parameters(dem),
                                      projection_parameters(dem)))
    slopes, _ = oracle.march_all_passes(segments, pyramids, tile_height=128,
                                        mask=oracle.PRODUCTION_MASK, **tile)
    expected = HorizonBuffers(slopes).degrees()
    finite = np.isfinite(expected)
    assert np.array_equal(finite, np.isfinite(got))
    error = np.abs(got[finite].astype(np.float64) - expected[finite])
    # Device and host FP64 segment fits differ by ulps; the horizons agree to
    # the 0.01 degree bar everywhere but a vanishing share of samples.
    assert np.mean(error > 0.01) <= 1e-4, float(np.max(error))
    assert np.median(error) == 0.0


def test_partial_tile_pads_outside_pixels_with_minus_fifty(synthetic_pair, cuda_session):
    primary, _ = synthetic_pair
    dems = [cuda_session.upload_dem_grid(primary)]
    raw = _tile(cuda_session, dems, tile_x=256, tile_y=256, azimuths=16, distance=20_000.0,
                observer=0.0)
    grid = raw.view("<f4").reshape(128, 128, 16)
    assert np.all(grid[:, 64:] == -50.0)   # columns beyond x = 320
    assert np.all(grid[64:, :] == -50.0)   # rows beyond y = 320
    # Rays of the last valid row/column that leave the DEM at once keep -inf,
    # as in the reference; everything inside has a horizon.
    assert not np.any(np.isnan(grid))
    assert np.all(np.isfinite(grid[:60, :60]))
    assert np.all(grid[:60, :60] > -50.0)


def test_compressed_tile_equals_encoding_of_the_raw_tile(synthetic_pair, cuda_session, codec):
    from lunarscout_b200.horizon import HorizonTileGenerator

    primary, _ = synthetic_pair
    with HorizonTileGenerator([primary], session=cuda_session) as generator:
        payload = bytes(generator.compute(256, 0, observer_elevation_m=2.0, compress=True,
                                          maximum_distance_m=30_000.0))
        degrees = generator.degrees(256, 0, observer_elevation_m=2.0,
                                    maximum_distance_m=30_000.0)
    assert payload == codec.encode(degrees)
    assert np.all(degrees.reshape(128, 128, AZ)[:, 64:] == -50.0)


def test_generate_horizons_writes_resumes_and_overwrites(tmp_path, synthetic_pair):
    from lunarscout_b200.dem_io import save_dem
    from lunarscout_b200.file_format import HorizonTileStore
    from lunarscout_b200.horizon import generate_horizons, generate_horizons_from_grids

    primary, _ = synthetic_pair
    small = type(primary)(np.ascontiguousarray(primary.elevation_m[:200, :150]),
                          primary.geo_transform, primary.projection)
    dem_path = save_dem(tmp_path / "site.npz", small)
    out = tmp_path / "horizons"
    events = []
    result = generate_horizons(out, [dem_path], observer_height_m=1.0, compress=False,
                               progress_callback=events.append)
    assert result == out.resolve()
    assert (tmp_path / "site.pyr.bin").is_file()
    store = HorizonTileStore(out)
    paths = sorted(out.rglob("*.bin"))
    assert [p.name for p in paths] == ["horizon_00000_00000_010.bin",
                                       "horizon_00000_00128_010.bin",
                                       "horizon_00128_00000_010.bin",
                                       "horizon_00128_00128_010.bin"]
    assert all(store.is_complete(p) for p in paths)
    assert events[0] == pytest.approx(0.1) and events[-1] == 1.0
    assert events == sorted(events)
    stamps = {p: p.stat().st_mtime_ns for p in paths}
    generate_horizons(out, [dem_path], observer_height_m=1.0, compress=False)
    assert {p: p.stat().st_mtime_ns for p in paths} == stamps      # resume: nothing rewritten

    # The in-memory entry on the same grid writes identical bytes.
    grid_out = tmp_path / "grid"
    generate_horizons_from_grids(grid_out, [small], observer_height_m=1.0, compress=False)
    for path in paths:
        twin = grid_out / path.relative_to(out)
        assert twin.read_bytes() == path.read_bytes()


@pytest.mark.parametrize("compress", [False, True])
def test_batched_generation_writes_the_per_tile_bytes(tmp_path, synthetic_pair, compress):
    from lunarscout_b200.file_format import HorizonTileStore
    from lunarscout_b200.horizon import generate_horizons_from_grids

    primary, _ = synthetic_pair
    small = type(primary)(np.ascontiguousarray(primary.elevation_m[:200, :300]),
                          primary.geo_transform, primary.projection)
    options = dict(observer_height_m=0.5, compress=compress, maximum_distance_m=40_000.0)
    generate_horizons_from_grids(tmp_path / "plain", [small], **options)
    generate_horizons_from_grids(tmp_path / "batched", [small], batch_tiles=4, **options)
    plain = sorted((tmp_path / "plain").rglob("horizon_*"))
    assert len(plain) == 6
    for path in plain:
        twin = tmp_path / "batched" / path.relative_to(tmp_path / "plain")
        assert twin.read_bytes() == path.read_bytes(), path.name
    generate_horizons_from_grids(tmp_path / "ladder", [small], batch_tiles=4,
                                 traversal="ladder", **options)
    ladder = sorted((tmp_path / "ladder").rglob("horizon_*"))
    assert [p.name for p in ladder] == [p.name for p in plain]
    assert all(HorizonTileStore.is_complete(p) for p in ladder)


def test_generator_tiles_fit_segments_on_the_float64_georeference(synthetic_pair, cuda_session):
    """The public generator uploads pyramids (whose georeference is float32)
    but fits segments with each DEM's float64 geotransform and projection:
    its tiles equal the device path fed the DemGrids themselves.  In float32
    the polar latitude origin -pi/2 rounds past the pole and moves the
    observers; at 1.5 m above the terrain that changed horizons by degrees."""
    from lunarscout_b200.horizon import HorizonTileGenerator

    primary, regional = synthetic_pair
    dems = [cuda_session.upload_dem_grid(primary), cuda_session.upload_dem_grid(regional)]
    tile = dict(tile_column=128, tile_row=128, tile_width=128, subpatch_size=8)
    with HorizonTileGenerator([primary, regional], session=cuda_session) as generator:
        got = generator.degrees(128, 128, observer_elevation_m=1.5, maximum_distance_m=100_000.0)
    segments = cuda_session.generate_segments(dems, azimuth_count=AZ,
                                              maximum_distance_m=100_000.0,
                                              observer_elevation_m=1.5, **tile)
    pyramids = [cuda_session.build_max_pyramid(primary), cuda_session.build_max_pyramid(regional)]
    slopes, _ = cuda_session.subpatch_hierarchical_all_passes(
        segments, pyramids, tile_height=128, observer_elevation_m=1.5, **tile)
    np.testing.assert_array_equal(got, cuda_session.slopes_to_degrees(slopes))
    for dem in dems:
        dem.close()
