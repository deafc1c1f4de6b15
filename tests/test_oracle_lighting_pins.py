"""Pin the lighting oracle against the reference (CPU only).

Fixtures: the reference's C# captures (BuilderSunFraction samples, ILGPU PSR
tiles) and the reference's own CPU backend run on a synthetic site
(tests/golden/make_golden.py).
"""

from __future__ import annotations

import hashlib

import numpy as np
import pytest

import oracle
from oracle import products
from conftest import load_golden


def synthetic_horizons(height=128, width=128):
    """Same deterministic horizon tile as tests/golden/make_golden.py."""
    az = np.radians(np.arange(1440, dtype=np.float64) * 0.25)
    y, x = np.mgrid[0:height, 0:width]
    phase = (0.05 * x + 0.03 * y)[..., None]
    level = (1.0 + 0.25 * (x - y))[..., None]
    h = level + 2.5 * np.sin(3.0 * az + phase) + 1.0 * np.sin(11.0 * az + 2.0 * phase)
    return np.ascontiguousarray(h, dtype=np.float32)


@pytest.fixture(scope="module")
def site():
    from lunarscout_b200 import synthetic

    arrays = load_golden("lighting_reference.npz")
    dem = synthetic.config1_dem()
    ty, tx, vh, vw = (int(v) for v in arrays["tile"])
    hours = arrays["hours"]
    return dict(dem=dem, arrays=arrays, tile=dict(tile_y=ty, tile_x=tx, valid_height=vh,
                                                  valid_width=vw),
                horizons=synthetic_horizons(), sun=synthetic.sun_vectors(hours),
                earth=synthetic.earth_vectors(hours))


def test_half_circle_constants():
    hc, photons = products.half_circle()
    expected = np.asarray([np.sqrt(64.0 - (7.5 - i) ** 2) / 8.0 * float(np.float32(0.27))
                           for i in range(16)], dtype=np.float32)
    np.testing.assert_array_equal(hc, expected)
    total = np.float32(0.0)
    for c in expected:
        total = np.float32(total + c)
    assert np.float32(photons) == np.float32(np.float32(2.0) * total)


def test_sun_fraction_matches_csharp_builder_bytes():
    arrays = load_golden("lighting_csharp.npz")
    checked = 0
    for index in range(3):
        horizon = arrays[f"lm{index}_horizon"]
        for az, el, byte, bits in arrays[f"lm{index}_samples"]:
            fraction = products.sun_fraction(horizon, az, el)[0]
            assert int(np.uint8(np.float32(255.0) * fraction)) == int(byte)
            # The reference's own float32 restatement sits within 3 ulp of
            # the C# fractions (MathF evaluation order); so does the oracle.
            ulp = abs(int(np.float32(fraction).view(np.int32)) - int(bits))
            assert ulp <= 3
            checked += 1
    assert checked == 24


def test_full_half_and_zero_disk_encode_255_127_0():
    horizon = np.zeros(1440, dtype=np.float32)
    got = [products.sun_fraction(horizon, 90.0, el)[0] for el in (1.0, 0.0, -1.0)]
    assert [int(np.uint8(np.float32(255) * g)) for g in got] == [255, 127, 0]


def test_lighting_oracle_is_bit_identical_to_the_reference_cpu_backend(site):
    fractions = products.lighting_tiles(site["dem"], site["horizons"], site["sun"],
                                        **site["tile"])
    np.testing.assert_array_equal(fractions, site["arrays"]["fractions"])
    margins = products.lighting_tiles(site["dem"], site["horizons"], site["earth"],
                                      margin=True, **site["tile"])
    np.testing.assert_array_equal(margins, site["arrays"]["margins"])
    assert 0.02 < np.mean((fractions > 0) & (fractions < 1)) < 0.98


def test_psr_vector_reduction_matches_reference(site):
    reduced, indices = products.reduce_sun_vectors(site["dem"], site["sun"])
    np.testing.assert_array_equal(indices, site["arrays"]["psr_reduced_indices"])
    np.testing.assert_array_equal(reduced, site["sun"][indices])


def test_psr_oracle_matches_reference(site):
    _, indices = products.reduce_sun_vectors(site["dem"], site["sun"])
    psr = products.psr_tile(site["dem"], site["horizons"], site["sun"][indices], **site["tile"])
    np.testing.assert_array_equal(psr, site["arrays"]["psr_reduced"])
    psr_all = products.psr_tile(site["dem"], site["horizons"], site["sun"], **site["tile"])
    np.testing.assert_array_equal(psr_all, site["arrays"]["psr_all"])
    assert 0 < np.count_nonzero(psr_all) < psr_all.size


def _csharp_psr_inputs(arrays, name):
    from lunarscout_b200.contract import DemGrid, ProjectionParameters

    x = np.arange(128, dtype=np.float64)[None, :]
    y = np.arange(128, dtype=np.float64)[:, None]
    dem = DemGrid(np.ascontiguousarray((x - y) * 0.1, dtype=np.float32),
                  np.ascontiguousarray(arrays["psr_geo_transform"]),
                  ProjectionParameters.from_array(arrays["psr_projection"]))
    pixel = np.arange(128 * 128, dtype=np.int32)[:, None]
    azimuth = np.arange(1440, dtype=np.int32)[None, :]
    if name == "constant_shadow":
        horizons = np.full((128 * 128, 1440), 0.3, dtype=np.float32)
    else:
        horizons = (np.float32(0.45) + np.float32(0.01) * (pixel % 23)
                    + np.float32(0.0001) * (azimuth % 17)).astype(np.float32)
        if name == "compressed_quantized_mixed":
            scaled = horizons * np.float32(32767.0 / 50.0)
            horizons = (np.floor(scaled + np.float32(0.5)).astype(np.int16)
                        * np.float32(50.0 / 32767.0)).astype(np.float32)
    return dem, horizons.reshape(128, 128, 1440)


def test_psr_oracle_matches_csharp_ilgpu_tiles():
    arrays = load_golden("lighting_csharp.npz")
    for index, name in enumerate(str(n) for n in arrays["psr_names"]):
        dem, horizons = _csharp_psr_inputs(arrays, name)
        got = products.psr_tile(dem, horizons, arrays[f"psr{index}_vectors"], tile_y=0, tile_x=0)
        np.testing.assert_array_equal(got, arrays[f"psr{index}_expected"], err_msg=name)


def _accepts(arrays, hours):
    bounds = arrays["interval_bounds_hours"]
    return np.stack([(hours >= lo) & (hours < hi) for lo, hi in bounds])


def _sample_hours(hours, stop):
    following = np.append(hours[1:], stop)
    return np.minimum(following, stop) - hours


def test_mission_duration_oracle_matches_reference(site):
    arrays = site["arrays"]
    hours = arrays["hours"]
    stop = float(arrays["evaluation_stop_hours"])
    accepts = _accepts(arrays, hours)
    durations = products.longest_duration(arrays["fractions"] >= np.float32(0.5),
                                          _sample_hours(hours, stop), accepts)
    np.testing.assert_array_equal(durations.astype(np.float32), arrays["durations_hours"])
    both = products.longest_duration(
        (arrays["fractions"] >= np.float32(0.5)) & (arrays["margins"] >= np.float32(0.0)),
        _sample_hours(hours, stop), accepts) / 24.0
    np.testing.assert_array_equal(both.astype(np.float32), arrays["durations_days_sun_earth"])


def test_cbin_codec_matches_reference_encoder():
    arrays = load_golden("codec_reference.npz")
    degrees = synthetic_horizons().reshape(-1, 1440) * np.float32(6.0)
    degrees[5, :7] = -np.inf
    degrees[9, 100:110] = 75.0
    payload = products.encode_tile(degrees)
    assert len(payload) == int(arrays["payload_size"])
    assert hashlib.sha256(payload).hexdigest() == str(arrays["payload_sha256"])
    decoded = products.decode_tile(payload)
    np.testing.assert_array_equal(decoded[[0, 5, 9, 777, 16383]], arrays["decoded_rows"])
    assert np.all(decoded[5, :7] == np.float32(-32767) * (np.float32(50.0) / np.float32(32767.0)))


def _reduction_cases():
    from lunarscout_b200 import synthetic

    arrays = load_golden("psr_reduction_reference.npz")
    dems = {"plain_year": synthetic.config1_dem, "site_three_years": synthetic.site_dem}
    for name, make in dems.items():
        first, last, step = arrays[f"{name}_hours"]
        hours = np.arange(first, last + 0.5 * step, step)
        yield name, make(), synthetic.sun_vectors(hours), arrays[f"{name}_indices"]


def test_psr_vector_reduction_matches_reference_on_long_tables():
    """One year hourly (8,761 vectors) and three years hourly (26,305
    vectors) against the reference's own reduce_sun_vectors_for_psr."""
    for name, dem, sun, expected in _reduction_cases():
        _, indices = products.reduce_sun_vectors(dem, sun)
        np.testing.assert_array_equal(indices, expected, err_msg=name)
