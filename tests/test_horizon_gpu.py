"""Horizon march, pyramid and segment generation on the B200 vs the oracle."""

from __future__ import annotations

import numpy as np
import pytest

import oracle
from oracle import segments as oseg
from conftest import load_golden
from test_oracle_pins import _path_error, halo_dems

pytestmark = pytest.mark.gpu

PROD = oracle.PRODUCTION_MASK


def _pyramid(dem):
    from lunarscout_b200.contract import PyramidArrays, map_parameters, projection_parameters

    mips, levels = oracle.build_pyramid(dem.elevation_m)
    return PyramidArrays(dem.elevation_m, mips, levels, map_parameters(dem),
                         projection_parameters(dem))


@pytest.fixture(scope="module")
def synthetic_pair():
    from lunarscout_b200.synthetic import SyntheticDemSpec, synthetic_dem

    primary = synthetic_dem(SyntheticDemSpec(512, 20.0, craters=40, seed=1))
    regional = synthetic_dem(SyntheticDemSpec(400, 240.0, sigma_m=1200.0, craters=0,
                                              tilt_m=2000.0, seed=1001))
    return primary, regional


def test_device_pyramid_matches_oracle_including_invalid_values(cuda_session):
    rng = np.random.default_rng(5)
    for height, width in ((513, 377), (41, 41), (5, 7), (1, 1), (1024, 3)):
        level0 = rng.normal(0.0, 300.0, size=(height, width)).astype(np.float32)
        level0.flat[rng.integers(0, level0.size, size=max(1, level0.size // 50))] = np.nan
        level0.flat[rng.integers(0, level0.size, size=max(1, level0.size // 70))] = np.inf
        level0.flat[rng.integers(0, level0.size, size=max(1, level0.size // 60))] = -25000.0

        class Dem:
            elevation_m = level0
            geo_transform = np.array((0, 20.0, 0, 0, 0, -20.0))

            class projection:
                radius_m, latitude_origin_rad, longitude_origin_rad = 1737400.0, -1.5707963, 0.0
                scale, false_easting_m, false_northing_m = 1.0, 0.0, 0.0

        got = cuda_session.build_max_pyramid(Dem)
        mips, levels = oracle.build_pyramid(level0)
        np.testing.assert_array_equal(got.levels, levels)
        np.testing.assert_array_equal(got.mips, mips)


def test_device_march_is_bit_identical_to_oracle_on_the_golden_case(production_case,
                                                                    cuda_session):
    arrays, pyramids = production_case
    common = dict(tile_column=20, tile_row=20, tile_width=1, tile_height=1, subpatch_size=8)
    gpu0 = cuda_session.subpatch_hierarchical_pass(arrays["segments"], pyramids[0],
                                                   pyramids[0], pass_index=0, **common)
    gpu1 = cuda_session.subpatch_hierarchical_pass(arrays["segments"], pyramids[0],
                                                   pyramids[1], pass_index=1, **common)
    for p, gpu in enumerate((gpu0, gpu1)):
        cpu, _ = oracle.march_pass(arrays["segments"], pyramids[0], pyramids[p],
                                   pass_index=p, mask=PROD, **common)
        np.testing.assert_array_equal(gpu, cpu)
    # Against the reference's C# capture: every value but the ray that the
    # superseded cell-exit cap changes (see test_oracle_pins).
    expected = arrays["csharp_per_dem_slopes"]
    diff = np.abs(np.stack([gpu0[0], gpu1[0]]) - expected)
    assert np.argwhere(diff > 3e-7).tolist() == [[1, 360]]
    final, seconds = cuda_session.subpatch_hierarchical_all_passes(
        arrays["segments"], pyramids, **common)
    cpu_final, _ = oracle.march_all_passes(arrays["segments"], pyramids, mask=PROD, **common)
    np.testing.assert_array_equal(final, cpu_final)
    assert len(seconds) == 2 and all(s >= 0 for s in seconds)


def test_device_march_full_tile_two_dems_bit_identical(synthetic_pair, cuda_session):
    primary, regional = synthetic_pair
    pyramids = [_pyramid(primary), _pyramid(regional)]
    tile = dict(tile_column=192, tile_row=192, tile_width=128, subpatch_size=8)
    segments = oseg.build_segments([primary, regional], azimuth_count=48,
                                   maximum_distance_m=200_000.0, observer_elevation_m=2.0,
                                   **tile)
    gpu, _ = cuda_session.subpatch_hierarchical_all_passes(
        segments, pyramids, tile_height=128, observer_elevation_m=2.0, **tile)
    cpu, _ = oracle.march_all_passes(segments, pyramids, tile_height=128,
                                     observer_elevation_m=2.0, mask=PROD, **tile)
    assert gpu.shape == (128 * 128, 48)
    np.testing.assert_array_equal(gpu, cpu)
    assert np.isfinite(gpu).all()


def test_partial_edge_tile_keeps_outside_pixels_at_sentinel(synthetic_pair, cuda_session):
    primary, _ = synthetic_pair
    pyramids = [_pyramid(primary)]
    tile = dict(tile_column=448, tile_row=480, tile_width=128, subpatch_size=8)
    segments = oseg.build_segments([primary], azimuth_count=16,
                                   maximum_distance_m=10_000.0, **tile)
    gpu, _ = cuda_session.subpatch_hierarchical_all_passes(segments, pyramids,
                                                           tile_height=128, **tile)
    cpu, _ = oracle.march_all_passes(segments, pyramids, tile_height=128, mask=PROD, **tile)
    np.testing.assert_array_equal(gpu, cpu)
    grid = gpu.reshape(128, 128, 16)
    assert np.all(np.isneginf(grid[:, 64:]))   # columns beyond x = 512
    assert np.all(np.isneginf(grid[32:, :]))   # rows beyond y = 512
    assert not np.any(np.isnan(grid))


def test_explicit_slope_carry_equals_all_passes(synthetic_pair, cuda_session):
    primary, regional = synthetic_pair
    pyramids = [_pyramid(primary), _pyramid(regional)]
    tile = dict(tile_column=0, tile_row=0, tile_width=32, subpatch_size=8)
    segments = oseg.build_segments([primary, regional], azimuth_count=24,
                                   maximum_distance_m=100_000.0, **tile)
    first = cuda_session.subpatch_hierarchical_pass(segments, pyramids[0], pyramids[0],
                                                    tile_height=32, pass_index=0, **tile)
    second = cuda_session.subpatch_hierarchical_pass(segments, pyramids[0], pyramids[1],
                                                     tile_height=32, pass_index=1,
                                                     slopes=first, **tile)
    combined, _ = cuda_session.subpatch_hierarchical_all_passes(segments, pyramids,
                                                                tile_height=32, **tile)
    np.testing.assert_array_equal(second, combined)


def test_device_segments_match_oracle(synthetic_pair, cuda_session):
    primary, regional = synthetic_pair
    dems = [cuda_session.upload_dem_grid(primary), cuda_session.upload_dem_grid(regional)]
    tile = dict(tile_column=128, tile_row=256, tile_width=128, subpatch_size=8)
    got = cuda_session.generate_segments(dems, azimuth_count=90,
                                         maximum_distance_m=200_000.0,
                                         observer_elevation_m=1.0, **tile)
    ref = oseg.build_segments([primary, regional], azimuth_count=90,
                              maximum_distance_m=200_000.0, observer_elevation_m=1.0, **tile)
    assert got.shape == ref.shape
    # FP64 transcendental results differ by ulps between CUDA and glibc; the
    # fitted paths agree far below the reference's 1e-5 px tolerance.
    assert _path_error(got, ref) < 1e-5
    np.testing.assert_allclose(got[..., 12:15], ref[..., 12:15], rtol=1e-6, atol=1e-6)
    np.testing.assert_allclose(got[..., 15:18], ref[..., 15:18], rtol=1e-4, atol=1e-9)


def test_device_segments_on_the_csharp_halo_fixture(cuda_session):
    arrays = load_golden("segments_halo.npz")
    tc, tr, tw, _th, sub, az, dist = (int(v) for v in arrays["config"])
    dems = [cuda_session.upload_dem(d.elevation_m, d.geo_transform, d.projection.as_array())
            for d in halo_dems(arrays)]
    got = cuda_session.generate_segments(dems, tile_column=tc, tile_row=tr, tile_width=tw,
                                         azimuth_count=az, maximum_distance_m=float(dist),
                                         subpatch_size=sub)
    assert _path_error(got, arrays["csharp_segments"]) < 1e-5
    assert _path_error(got, arrays["reference_numba_segments"]) < 1e-5


def test_degrees_conversion_matches_host_contract(cuda_session):
    from lunarscout_b200.contract import HorizonBuffers

    rng = np.random.default_rng(3)
    slopes = rng.normal(0, 0.2, size=(64, 1440)).astype(np.float32)
    slopes[3, 5] = -np.inf
    got = cuda_session.slopes_to_degrees(slopes)
    expected = HorizonBuffers(slopes).degrees()
    assert np.isneginf(got[3, 5])
    np.testing.assert_allclose(got, expected, rtol=0, atol=1e-5)


def test_device_march_reproduces_the_reference_numba_cuda_slopes(cuda_session):
    """The drop-in on the same inputs as the reference's own Numba-CUDA
    kernel run on a B200 (tests/golden/numba_cuda_b200.npz: two DEM passes,
    16,384 pixels x 12 azimuths): every slope bit for bit."""
    from test_oracle_pins import _numba_case

    arrays, pyramids, common = _numba_case()
    gpu, _ = cuda_session.subpatch_hierarchical_all_passes(
        arrays["segments"], pyramids, tile_width=128, tile_height=128, subpatch_size=8,
        **common)
    np.testing.assert_array_equal(gpu, arrays["slopes"])
