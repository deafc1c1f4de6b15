"""Lightmap (fraction, bytes, margin) and PSR on the B200 vs the oracle.

Tolerances are the path's accuracy targets: sun fraction within 1e-4 absolute of the
reference CPU backend; PSR bit-exact except a counted band of pixels whose
peak (sun centre - horizon) lies within 1e-4 deg of the -0.2725 deg limb
threshold.  Differences come only from CUDA's atan2f vs glibc's.
"""

from __future__ import annotations

import numpy as np
import pytest

from oracle import products
from conftest import load_golden
from test_oracle_lighting_pins import _csharp_psr_inputs, synthetic_horizons

pytestmark = pytest.mark.gpu

FRACTION_TOL = 1e-4
MARGIN_TOL = 1e-4
BAND_DEG = 1e-4


@pytest.fixture(scope="module")
def lighting_session():
    from lunarscout_b200.lightmap_cuda import LightmapCudaSession

    session = LightmapCudaSession(time_batch_size=32)
    yield session
    session.close()


@pytest.fixture(scope="module")
def psr_session():
    from lunarscout_b200.psr_cuda import PsrCudaSession

    session = PsrCudaSession()
    yield session
    session.close()


@pytest.fixture(scope="module")
def site():
    from lunarscout_b200 import synthetic

    hours = synthetic.hours_between("2029-01-01T00", "2029-02-01T00", 6.0)
    return dict(dem=synthetic.config1_dem(), horizons=synthetic_horizons(),
                sun=synthetic.sun_vectors(hours), earth=synthetic.earth_vectors(hours),
                tile=dict(tile_y=448, tile_x=448, valid_height=40, valid_width=48))


def test_sun_fraction_kernel_is_bit_identical_on_csharp_samples(lighting_session):
    arrays = load_golden("lighting_csharp.npz")
    for index in range(3):
        horizon = arrays[f"lm{index}_horizon"]
        samples = arrays[f"lm{index}_samples"]
        rows = np.repeat(horizon[None, :], len(samples), axis=0)
        gpu = lighting_session.sun_fraction(rows, samples[:, 0], samples[:, 1])
        cpu = products.sun_fraction(rows, samples[:, 0], samples[:, 1])
        np.testing.assert_array_equal(gpu, cpu)
        np.testing.assert_array_equal((np.float32(255) * gpu).astype(np.uint8),
                                      samples[:, 2].astype(np.uint8))


def test_fraction_tiles_match_reference_cpu_backend(lighting_session, site):
    tiles = list(lighting_session.iter_patch_fraction_tiles(
        site["dem"], site["horizons"], site["sun"], **site["tile"]))
    assert len(tiles) == len(site["sun"])
    assert tiles[0].shape == (40, 48) and tiles[0].dtype == np.float32
    gpu = np.stack(tiles)
    cpu = products.lighting_tiles(site["dem"], site["horizons"], site["sun"], **site["tile"])
    error = np.abs(gpu - cpu)
    assert error.max() <= FRACTION_TOL, error.max()
    assert np.mean(gpu == cpu) > 0.9


def test_byte_tiles_differ_by_at_most_one_count(lighting_session, site):
    gpu = np.stack(list(lighting_session.iter_patch_tiles(
        site["dem"], site["horizons"], site["sun"], **site["tile"])))
    assert gpu.dtype == np.uint8
    cpu = products.encode_fraction_bytes(
        products.lighting_tiles(site["dem"], site["horizons"], site["sun"], **site["tile"]))
    diff = np.abs(gpu.astype(np.int16) - cpu.astype(np.int16))
    assert diff.max() <= 1
    assert np.count_nonzero(diff) <= 0.001 * diff.size


def test_margin_tiles_match_reference_cpu_backend(lighting_session, site):
    gpu = np.stack(list(lighting_session.iter_patch_margin_tiles(
        site["dem"], site["horizons"], site["earth"], **site["tile"])))
    cpu = products.lighting_tiles(site["dem"], site["horizons"], site["earth"], margin=True,
                                  **site["tile"])
    assert np.abs(gpu - cpu).max() <= MARGIN_TOL


def test_full_tile_and_time_blocks_longer_than_one_launch(lighting_session, site):
    from lunarscout_b200 import synthetic

    hours = synthetic.hours_between("2029-01-01T00", "2029-03-15T00", 1.0)[:1500]
    vectors = synthetic.sun_vectors(hours)
    tile = dict(tile_y=128, tile_x=256)
    gpu = np.stack(list(lighting_session.iter_patch_fraction_tiles(
        site["dem"], site["horizons"], vectors, **tile)))
    assert gpu.shape == (1500, 128, 128)
    picks = np.array([0, 1, 31, 32, 1023, 1024, 1499])
    cpu = products.lighting_tiles(site["dem"], site["horizons"], vectors[picks], **tile)
    assert np.abs(gpu[picks] - cpu).max() <= FRACTION_TOL


def test_psr_matches_oracle_outside_the_threshold_band(psr_session, site):
    _, indices = products.reduce_sun_vectors(site["dem"], site["sun"])
    reduced = site["sun"][indices]
    gpu = psr_session.compute_patch(site["dem"], site["horizons"], reduced, **site["tile"])
    cpu = products.psr_tile(site["dem"], site["horizons"], reduced, **site["tile"])
    peak = products.psr_peak_margin(site["dem"], site["horizons"], reduced, **site["tile"])
    band = np.abs(peak - products.PSR_LIMB_THRESHOLD) < BAND_DEG
    mismatched = gpu != cpu
    assert not np.any(mismatched & ~band), np.argwhere(mismatched & ~band)[:5]
    assert 0 < np.count_nonzero(gpu == 255) < gpu.size


def test_psr_matches_csharp_ilgpu_tiles(psr_session):
    from lunarscout_b200.contract import DemGrid

    arrays = load_golden("lighting_csharp.npz")
    for index, name in enumerate(str(n) for n in arrays["psr_names"]):
        dem, horizons = _csharp_psr_inputs(arrays, name)
        vectors = arrays[f"psr{index}_vectors"]
        gpu = psr_session.compute_patch(dem, horizons, vectors, tile_y=0, tile_x=0)
        expected = arrays[f"psr{index}_expected"]
        peak = products.psr_peak_margin(dem, horizons, vectors, tile_y=0, tile_x=0)
        band = np.abs(peak - products.PSR_LIMB_THRESHOLD) < BAND_DEG
        assert not np.any((gpu != expected) & ~band), name


def test_psr_pinned_buffer_and_validation(psr_session, site):
    buffer = psr_session.allocate_pinned_horizon_buffer()
    assert buffer.shape == (128, 128, 1440) and buffer.dtype == np.float32
    buffer[...] = site["horizons"]
    out = psr_session.compute_patch(site["dem"], buffer, site["sun"][:10], tile_y=0, tile_x=0)
    assert out.shape == (128, 128)
    with pytest.raises(ValueError):
        psr_session.compute_patch(site["dem"], buffer, site["sun"][:10], tile_y=500, tile_x=0)
    with pytest.raises(ValueError):
        psr_session.compute_patch(site["dem"], buffer[:64], site["sun"][:10], tile_y=0, tile_x=0)


def _duration_inputs(hours, stop, bounds):
    following = np.append(hours[1:], stop)
    sample_hours = np.minimum(following, stop) - hours
    accepts = np.stack([(hours >= lo) & (hours < hi) for lo, hi in bounds])
    windows = np.array([[np.searchsorted(hours, lo, "left"), np.searchsorted(hours, hi, "left")]
                        for lo, hi in bounds], dtype=np.int32)
    return sample_hours, accepts, windows


@pytest.mark.parametrize("stop", [750.0, 746.5])
def test_mission_durations_reduce_the_device_conditions_exactly(lighting_session, site, stop):
    hours = np.arange(len(site["sun"]), dtype=np.float64) * 6.0
    bounds = [(0.0, 168.0), (168.0, 336.0), (336.0, 504.0), (504.0, 744.0), (100.0, 101.0)]
    sample_hours, accepts, windows = _duration_inputs(hours, stop, bounds)
    fractions = np.stack(list(lighting_session.iter_patch_fraction_tiles(
        site["dem"], site["horizons"], site["sun"], **site["tile"])))
    margins = np.stack(list(lighting_session.iter_patch_margin_tiles(
        site["dem"], site["horizons"], site["earth"], **site["tile"])))
    got = lighting_session.mission_durations(site["dem"], site["horizons"], site["sun"],
                                             sample_hours=sample_hours, start_windows=windows,
                                             **site["tile"])
    expected = products.longest_duration(fractions >= np.float32(0.5), sample_hours, accepts)
    np.testing.assert_array_equal(got, expected.astype(np.float32))
    assert got.shape == (len(bounds), 40, 48) and got.max() > 0.0
    both = lighting_session.mission_durations(
        site["dem"], site["horizons"], site["sun"], earth_vectors_m=site["earth"], days=True,
        sample_hours=sample_hours, start_windows=windows, **site["tile"])
    expected = products.longest_duration(
        (fractions >= np.float32(0.5)) & (margins >= np.float32(0.0)), sample_hours,
        accepts) / 24.0
    np.testing.assert_array_equal(both, expected.astype(np.float32))


def test_mission_durations_against_the_reference_cpu_chain(lighting_session, site):
    hours = np.arange(len(site["sun"]), dtype=np.float64) * 6.0
    bounds = [(0.0, 240.0), (240.0, 480.0), (480.0, 744.0)]
    sample_hours, accepts, windows = _duration_inputs(hours, 750.0, bounds)
    got = lighting_session.mission_durations(site["dem"], site["horizons"], site["sun"],
                                             sample_hours=sample_hours, start_windows=windows,
                                             **site["tile"])
    cpu = products.lighting_tiles(site["dem"], site["horizons"], site["sun"], **site["tile"])
    expected = products.longest_duration(cpu >= np.float32(0.5), sample_hours, accepts)
    # Fractions differ from the CPU backend by <= 1e-4 (atan2f); a condition
    # can flip only for fractions within that of the threshold.
    differ = got != expected.astype(np.float32)
    near = (np.abs(cpu - np.float32(0.5)) <= 1e-4).any(axis=0)
    assert np.all(near[differ.any(axis=0)])
    assert differ.mean() <= 0.01


@pytest.fixture(scope="module")
def haven(lighting_session, site):
    from datetime import datetime, timedelta, timezone

    from lunarscout_b200 import synthetic
    from lunarscout_b200.safe_haven import month_bands, month_indices

    hours = synthetic.hours_between("2029-01-20T00", "2029-04-10T00", 3.0)
    start = datetime(2029, 1, 20, tzinfo=timezone.utc)
    times = [start + timedelta(hours=float(h)) for h in hours]
    bands = month_bands(times)
    sun, earth = synthetic.sun_vectors(hours), synthetic.earth_vectors(hours)
    fractions = np.stack(list(lighting_session.iter_patch_fraction_tiles(
        site["dem"], site["horizons"], sun, **site["tile"])))
    margins = np.stack(list(lighting_session.iter_patch_margin_tiles(
        site["dem"], site["horizons"], earth, **site["tile"])))
    return dict(times=times, bands=bands, months=month_indices(times, bands), sun=sun,
                earth=earth, fractions=fractions, margins=margins)


def test_safe_haven_reduces_the_device_streams_exactly(lighting_session, site, haven):
    assert len(haven["bands"]) == 4
    cases = [(0.2, 2.0), (0.5, float(np.quantile(haven["margins"], 0.3)))]
    for sunlight, earth_deg in cases:
        got = lighting_session.safe_haven_durations(
            site["dem"], site["horizons"], haven["sun"], haven["earth"],
            month_index_of=haven["months"], band_count=len(haven["bands"]),
            time_step_hours=3.0, sunlight_threshold=sunlight, earth_threshold_deg=earth_deg,
            **site["tile"])
        expected = products.safe_haven(haven["fractions"], haven["margins"], haven["months"],
                                       len(haven["bands"]), sunlight_threshold=sunlight,
                                       earth_threshold_deg=earth_deg, time_step_hours=3.0)
        got = np.stack(got)
        assert got.shape == (4, 40, 48)
        np.testing.assert_array_equal(got, expected)
    assert np.isnan(got).any() and (got[np.isfinite(got)] > 0).any()


def test_safe_haven_unordered_months_and_the_patch_helper(lighting_session, site, haven):
    from lunarscout_b200.safe_haven import safe_haven_patch

    months = haven["months"].copy()
    months[100:300] = months[100:300][::-1]
    months[::7] = -1
    earth_deg = float(np.quantile(haven["margins"], 0.5))
    got = np.stack(lighting_session.safe_haven_durations(
        site["dem"], site["horizons"], haven["sun"], haven["earth"], month_index_of=months,
        band_count=4, time_step_hours=0.75, sunlight_threshold=0.5,
        earth_threshold_deg=earth_deg, **site["tile"]))
    expected = products.safe_haven(haven["fractions"], haven["margins"], months, 4,
                                   sunlight_threshold=0.5, earth_threshold_deg=earth_deg,
                                   time_step_hours=0.75)
    np.testing.assert_array_equal(got, expected)
    bands, durations = safe_haven_patch(lighting_session, site["dem"], site["horizons"],
                                        haven["times"], haven["sun"], haven["earth"],
                                        time_step_hours=3.0, **site["tile"])
    assert bands == haven["bands"]
    expected = products.safe_haven(haven["fractions"], haven["margins"], haven["months"], 4,
                                   sunlight_threshold=0.2, earth_threshold_deg=2.0,
                                   time_step_hours=3.0)
    np.testing.assert_array_equal(np.stack(durations), expected)


def test_safe_haven_validation(lighting_session, site, haven):
    common = dict(month_index_of=haven["months"], band_count=4, time_step_hours=3.0,
                  **site["tile"])
    args = (site["dem"], site["horizons"], haven["sun"], haven["earth"])
    for bad in (dict(sunlight_threshold=1.5), dict(earth_threshold_deg=float("nan")),
                dict(time_step_hours=0.0), dict(band_count=0),
                dict(month_index_of=haven["months"][:-1]),
                dict(month_index_of=np.full_like(haven["months"], 4))):
        with pytest.raises(ValueError):
            lighting_session.safe_haven_durations(*args, **{**common, **bad})
    with pytest.raises(ValueError):
        lighting_session.safe_haven_durations(site["dem"], site["horizons"], haven["sun"],
                                              haven["earth"][:-1], **common)


def test_earth_visibility_counts_the_device_margins_exactly(lighting_session, site, haven):
    for threshold in (0.0, float(np.quantile(haven["margins"], 0.4))):
        got = lighting_session.earth_visibility_fraction(
            site["dem"], site["horizons"], haven["earth"], threshold_deg=threshold,
            **site["tile"])
        np.testing.assert_array_equal(got, products.earth_visibility(haven["margins"],
                                                                     threshold))
    assert got.shape == (40, 48) and 0.0 < got.mean() < 1.0
    with pytest.raises(ValueError):
        lighting_session.earth_visibility_fraction(site["dem"], site["horizons"],
                                                   haven["earth"], threshold_deg=float("inf"),
                                                   **site["tile"])


def test_earth_visibility_against_the_reference_cpu_margins(lighting_session, site):
    golden = load_golden("lighting_reference.npz")
    got = lighting_session.earth_visibility_fraction(site["dem"], site["horizons"],
                                                     site["earth"], **site["tile"])
    expected = products.earth_visibility(golden["margins"], 0.0)
    # Margins agree with the reference CPU backend within 1e-4 deg; a step
    # can flip only where its margin lies within that of the threshold.
    flips = np.count_nonzero(np.abs(golden["margins"]) <= MARGIN_TOL, axis=0)
    assert np.all(np.abs(got - expected) * len(golden["margins"]) <= flips + 1e-3)


def test_device_psr_vector_reduction_equals_the_oracle(psr_session, site):
    """The device reduction (ls200_psr_reduce_vectors) against the oracle on
    the 125-step table and against the reference's own indices on one year
    (8,761) and three years (26,305) of hourly vectors."""
    from lunarscout_b200.psr_cuda import reduce_sun_vectors_for_psr
    from test_oracle_lighting_pins import _reduction_cases

    reduced, indices = psr_session.reduce_sun_vectors(site["dem"], site["sun"])
    _, expected = products.reduce_sun_vectors(site["dem"], site["sun"])
    np.testing.assert_array_equal(indices, expected)
    np.testing.assert_array_equal(reduced, site["sun"][expected])
    for name, dem, sun, expected in _reduction_cases():
        _, indices = reduce_sun_vectors_for_psr(dem, sun)
        np.testing.assert_array_equal(indices, expected, err_msg=name)
    with pytest.raises(ValueError):
        psr_session.reduce_sun_vectors(site["dem"], np.zeros((0, 3)))
    with pytest.raises(ValueError):
        psr_session.reduce_sun_vectors(site["dem"], np.full((4, 3), np.nan))
