"""The skip-ladder traversal of the batched march (oracle flag OPT_LADDER):
it only removes steps, it is the reference traversal where it does not act,
and its distance from the FP64 restatement matches the reference traversal's
(on the 512 x 512 plain configuration and a site-scale tile pair)."""

from __future__ import annotations

import numpy as np
import pytest

import oracle
from oracle import segments as oseg


def _pyramid(dem):
    from lunarscout_b200.contract import PyramidArrays, map_parameters, projection_parameters

    mips, levels = oracle.build_pyramid(dem.elevation_m)
    return PyramidArrays(dem.elevation_m, mips, levels, map_parameters(dem),
                         projection_parameters(dem))


def _degrees(slopes):
    return np.degrees(np.arctan(np.asarray(slopes, dtype=np.float64)))


@pytest.fixture(scope="module")
def plain_case():
    from lunarscout_b200 import synthetic

    dem = synthetic.config1_dem()
    tile = dict(tile_column=192, tile_row=192)
    segments = oseg.build_segments([dem], tile_width=128, azimuth_count=1440,
                                   maximum_distance_m=10_000.0, subpatch_size=8, **tile)
    rng = np.random.default_rng(4)
    rays = dict(pixels=rng.integers(0, 16384, 6000).astype(np.int32),
                azimuths=rng.integers(0, 1440, 6000).astype(np.int32))
    return segments, [_pyramid(dem)], tile, rays


def test_ladder_acting_nowhere_is_the_reference_traversal(plain_case):
    segments, pyramids, tile, rays = plain_case
    plain, counts = oracle.march_all_passes(segments, pyramids, **tile, **rays)
    # 10 km rays never reach the 15 km threshold.
    idle, idle_counts = oracle.march_all_passes(segments, pyramids, mask=oracle.ladder_mask(0, 15),
                                                **tile, **rays)
    np.testing.assert_array_equal(idle, plain)
    assert idle_counts == counts


def test_ladder_saves_visits_and_keeps_the_fp64_distance(plain_case):
    segments, pyramids, tile, rays = plain_case
    plain, (plain_visits, _) = oracle.march_all_passes(segments, pyramids, **tile, **rays)
    ladder, (ladder_visits, _) = oracle.march_all_passes(
        segments, pyramids, mask=oracle.ladder_mask(0, 1), **tile, **rays)
    fp64, _ = oracle.march_all_passes(segments, pyramids, precision="f64", **tile, **rays)
    assert ladder_visits < 0.7 * plain_visits
    d_plain, d_ladder, d_64 = _degrees(plain), _degrees(ladder), _degrees(fp64)
    finite = np.isfinite(d_plain)
    assert np.array_equal(finite, np.isfinite(d_ladder))
    to_plain = np.abs(d_ladder[finite] - d_plain[finite])
    assert np.quantile(to_plain, 0.999) < 1e-3 and to_plain.max() < 0.05
    err_plain = np.abs(d_plain[finite] - d_64[finite])
    err_ladder = np.abs(d_ladder[finite] - d_64[finite])
    assert np.quantile(err_ladder, 0.999) <= np.quantile(err_plain, 0.999) + 1e-3
    assert err_ladder.max() <= err_plain.max() + 0.01


def test_ladder_on_a_site_tile_with_a_regional_pass():
    from lunarscout_b200.synthetic import SyntheticDemSpec, synthetic_dem

    site = synthetic_dem(SyntheticDemSpec(1024, 5.0, craters=150, crater_max_m=4000.0, seed=2))
    regional = synthetic_dem(SyntheticDemSpec(600, 240.0, sigma_m=1200.0, craters=0,
                                              tilt_m=2000.0, seed=1002))
    tile = dict(tile_column=448, tile_row=448)
    segments = oseg.build_segments([site, regional], tile_width=128, azimuth_count=1440,
                                   maximum_distance_m=60_000.0, subpatch_size=8, **tile)
    pyramids = [_pyramid(site), _pyramid(regional)]
    rng = np.random.default_rng(5)
    rays = dict(pixels=rng.integers(0, 16384, 3000).astype(np.int32),
                azimuths=rng.integers(0, 1440, 3000).astype(np.int32))
    plain, (plain_visits, _) = oracle.march_all_passes(segments, pyramids, **tile, **rays)
    ladder, (ladder_visits, _) = oracle.march_all_passes(
        segments, pyramids, mask=oracle.ladder_mask(0, 1), **tile, **rays)
    fp64, _ = oracle.march_all_passes(segments, pyramids, precision="f64", **tile, **rays)
    assert ladder_visits < 0.5 * plain_visits
    finite = np.isfinite(plain)
    err_plain = np.abs(_degrees(plain) - _degrees(fp64))[finite]
    err_ladder = np.abs(_degrees(ladder) - _degrees(fp64))[finite]
    assert np.quantile(err_ladder, 0.999) <= np.quantile(err_plain, 0.999) + 1e-3
