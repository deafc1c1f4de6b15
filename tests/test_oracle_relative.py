"""The relative FP32 arithmetic of the march (oracle flag OPT_RELATIVE)
against the FP64 restatement of the reference march.

The reference march rounds absolute quantities in FP32: pixel coordinates
(an ulp is 3e-5 px at 512 px, 5e-4 px at 4096 px), the interpolated segment
start, absolute heights and R + height.  Its first level-0 sample lies 1 m
from the observer, where a 0.1 mm height error is already 0.006 deg.  The
relative arithmetic marches the same algorithm on an integer local origin
plus small offsets, with heights taken relative to the observer's z before
interpolation, and stays within ~1e-4 deg of the FP64 march on the plain
512 x 512 configuration (20 m, 10 km rays, one centred tile).  The GPU
kernels' relative traversals are bit-identical to this restatement
(tests/test_march_sites_gpu.py).
"""

from __future__ import annotations

import numpy as np
import pytest

import oracle
from oracle import segments as oseg


@pytest.fixture(scope="module")
def plain_case():
    from lunarscout_b200 import synthetic
    from lunarscout_b200.contract import PyramidArrays, map_parameters, projection_parameters

    dem = synthetic.config1_dem()
    mips, levels = oracle.build_pyramid(dem.elevation_m)
    pyramid = PyramidArrays(dem.elevation_m, mips, levels, map_parameters(dem),
                            projection_parameters(dem))
    segments = oseg.build_segments([dem], tile_column=192, tile_row=192, tile_width=128,
                                   azimuth_count=1440, maximum_distance_m=10_000.0,
                                   observer_elevation_m=0.0)
    rng = np.random.default_rng(21)
    pixels = rng.integers(0, 128 * 128, 4000).astype(np.int32)
    azimuths = rng.integers(0, 1440, 4000).astype(np.int32)
    common = dict(tile_column=192, tile_row=192, observer_elevation_m=0.0, pixels=pixels,
                  azimuths=azimuths)
    fp64, _ = oracle.march_all_passes(segments, [pyramid], precision="f64", **common)
    return segments, pyramid, common, fp64


def _error_deg(slopes, fp64):
    a = np.degrees(np.arctan(np.asarray(slopes, dtype=np.float64)))
    b = np.degrees(np.arctan(fp64))
    assert np.array_equal(np.isfinite(a), np.isfinite(b))
    finite = np.isfinite(b)
    return np.abs(a[finite] - b[finite])


def test_relative_arithmetic_meets_the_horizon_gate(plain_case):
    segments, pyramid, common, fp64 = plain_case
    relative, _ = oracle.march_all_passes(
        segments, [pyramid], mask=oracle.PRODUCTION_MASK | oracle.OPT_RELATIVE, **common)
    error = _error_deg(relative, fp64)
    assert error.max() <= 0.01, float(error.max())
    assert np.quantile(error, 0.999) <= 1e-3, float(np.quantile(error, 0.999))


def test_reference_arithmetic_is_further_from_fp64(plain_case):
    segments, pyramid, common, fp64 = plain_case
    production, _ = oracle.march_all_passes(segments, [pyramid], **common)
    relative, _ = oracle.march_all_passes(
        segments, [pyramid], mask=oracle.PRODUCTION_MASK | oracle.OPT_RELATIVE, **common)
    assert _error_deg(production, fp64).max() > 5 * _error_deg(relative, fp64).max()


def test_relative_ladder_stays_within_the_gate_at_p999(plain_case):
    segments, pyramid, common, fp64 = plain_case
    ladder, _ = oracle.march_all_passes(
        segments, [pyramid], mask=oracle.ladder_mask(0, 1) | oracle.OPT_RELATIVE, **common)
    error = _error_deg(ladder, fp64)
    # The ladder samples other positions after a skip, so single rays may
    # move by a sampling step; the bulk stays at the arithmetic's level.
    assert np.quantile(error, 0.999) <= 2e-3, float(np.quantile(error, 0.999))


def test_relative_mode_changes_nothing_in_fp64(plain_case):
    segments, pyramid, common, fp64 = plain_case
    relative64, _ = oracle.march_all_passes(
        segments, [pyramid], precision="f64", mask=oracle.PRODUCTION_MASK | oracle.OPT_RELATIVE,
        **common)
    assert np.abs(np.degrees(np.arctan(relative64)) - np.degrees(np.arctan(fp64))).max() < 1e-9
