"""The fused horizon -> lighting chain on the B200: its tiles are the
generator's bytes, and each product equals the per-patch session call fed
the same horizons (host round trip) — the chain only removes the round trip."""

from __future__ import annotations

from datetime import datetime, timedelta, timezone

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def chain_case():
    from lunarscout_b200 import synthetic
    from lunarscout_b200.chain import ProductChain
    from lunarscout_b200.pipeline import enumerate_patches
    from lunarscout_b200.synthetic import SyntheticDemSpec, synthetic_dem

    dem = synthetic_dem(SyntheticDemSpec(320, 20.0, craters=30, seed=5))
    small = type(dem)(np.ascontiguousarray(dem.elevation_m[:200, :300]), dem.geo_transform,
                      dem.projection)
    chain = ProductChain([small], maximum_distance_m=40_000.0, observer_elevation_m=0.5)
    patches = enumerate_patches(small.width, small.height)
    batch = chain.march(patches)
    hours = synthetic.hours_between("2029-01-25T00", "2029-03-05T00", 6.0)
    yield dict(chain=chain, dem=small, patches=patches, batch=batch, hours=hours,
               sun=synthetic.sun_vectors(hours), earth=synthetic.earth_vectors(hours))
    chain.close()


def _host(batch, i):
    """The horizons a .cbin round trip would hand the sessions at -inf (-50),
    unquantized."""
    h = batch.horizons[i].view(128, 128, 1440).cpu().numpy()
    return np.where(np.isneginf(h), np.float32(-50.0), h)


def _tile(patch):
    return dict(tile_y=patch.tile_y, tile_x=patch.tile_x, valid_height=patch.height,
                valid_width=patch.width)


@pytest.mark.parametrize("compress", [False, True])
def test_chain_tiles_are_the_generator_bytes(tmp_path, chain_case, compress):
    from lunarscout_b200.file_format import HorizonTileStore, TileCodec
    from lunarscout_b200.horizon import generate_horizons_from_grids

    chain, batch = chain_case["chain"], chain_case["batch"]
    assert len(batch) == 6 and any(p.width < 128 or p.height < 128 for p in batch.patches)
    generate_horizons_from_grids(tmp_path / "generator", [chain_case["dem"]],
                                 observer_height_m=0.5, compress=compress,
                                 maximum_distance_m=40_000.0)
    codec = TileCodec(context=chain.session.context)
    try:
        store = HorizonTileStore(tmp_path / "chain", codec=codec)
        chain.write_tiles(batch, store, compress=compress)
        chain.wait_for_writes()
    finally:
        codec.close()
    written = sorted((tmp_path / "generator").rglob("horizon_*"))
    assert len(written) == 6
    for path in written:
        twin = tmp_path / "chain" / path.relative_to(tmp_path / "generator")
        assert twin.read_bytes() == path.read_bytes(), path.name


def test_chain_products_equal_the_per_patch_sessions(chain_case):
    from lunarscout_b200.lightmap_cuda import LightmapCudaSession
    from lunarscout_b200.psr_cuda import PsrCudaSession
    from lunarscout_b200.safe_haven import month_bands, month_indices

    chain, batch, dem = chain_case["chain"], chain_case["batch"], chain_case["dem"]
    sun, earth, hours = chain_case["sun"], chain_case["earth"], chain_case["hours"]
    lighting = LightmapCudaSession(time_batch_size=32)
    psr_session = PsrCudaSession()
    start = datetime(2029, 1, 25, tzinfo=timezone.utc)
    times = [start + timedelta(hours=float(h)) for h in hours]
    bands = month_bands(times)
    months = month_indices(times, bands)
    sample_hours = np.full(len(hours), 6.0)
    windows = np.array([[0, 40], [40, 100], [100, len(hours)]], dtype=np.int32)
    try:
        fractions = chain.sun_fractions(batch, sun).cpu().numpy()
        encoded = chain.sun_fraction_bytes(batch, sun).cpu().numpy()
        psr = chain.psr(batch, sun, reduce=False)
        missions = chain.mission_durations(batch, sun, sample_hours=sample_hours,
                                           start_windows=windows, earth_vectors_m=earth)
        havens = chain.safe_haven(batch, sun, earth, month_index_of=months,
                                  band_count=len(bands), time_step_hours=6.0,
                                  sunlight_threshold=0.5, earth_threshold_deg=1.0)
        visible = chain.earth_visibility(batch, earth)
        for i, patch in enumerate(batch.patches):
            horizons, tile = _host(batch, i), _tile(patch)
            h, w = patch.height, patch.width
            expected = np.stack(list(lighting.iter_patch_fraction_tiles(dem, horizons, sun,
                                                                        **tile)))
            got = fractions[i].reshape(len(sun), 128, 128)[:, :h, :w]
            np.testing.assert_array_equal(got, expected)
            expected = np.stack(list(lighting.iter_patch_tiles(dem, horizons, sun, **tile)))
            np.testing.assert_array_equal(encoded[i].reshape(len(sun), 128, 128)[:, :h, :w],
                                          expected)
            np.testing.assert_array_equal(psr[i], psr_session.compute_patch(dem, horizons,
                                                                            sun, **tile))
            np.testing.assert_array_equal(missions[i], lighting.mission_durations(
                dem, horizons, sun, sample_hours=sample_hours, start_windows=windows,
                earth_vectors_m=earth, **tile))
            np.testing.assert_array_equal(havens[i], np.stack(
                lighting.safe_haven_durations(dem, horizons, sun, earth, month_index_of=months,
                                              band_count=len(bands), time_step_hours=6.0,
                                              sunlight_threshold=0.5, earth_threshold_deg=1.0,
                                              **tile)))
            np.testing.assert_array_equal(visible[i], lighting.earth_visibility_fraction(
                dem, horizons, earth, **tile))
        assert any(float(m.max()) > 0.0 for m in missions)
    finally:
        lighting.close()
        psr_session.close()


def test_chain_psr_is_the_reference_product_on_the_oracle(chain_case):
    """chain.psr reduces the vectors over the DEM (as the PSR pipeline does)
    and evaluates every patch against them: equal to the oracle's reduction
    followed by the oracle's PSR, outside the counted 1e-4 deg band around the
    limb threshold."""
    from oracle import products

    from lunarscout_b200 import synthetic

    chain, batch, dem = chain_case["chain"], chain_case["batch"], chain_case["dem"]
    # A year of hourly vectors: many share a viewpoint's azimuth bin.
    sun = synthetic.sun_vectors(synthetic.hours_between("2030-01-01T00", "2031-01-01T00", 1.0))
    reduced, indices = chain.reduced_sun_vectors(sun)
    _, expected_indices = products.reduce_sun_vectors(dem, sun)
    np.testing.assert_array_equal(indices, expected_indices)
    np.testing.assert_array_equal(reduced, sun[expected_indices])
    assert len(indices) < len(sun) // 2
    psr = chain.psr(batch, sun)
    band_pixels = 0
    for i, patch in enumerate(batch.patches):
        horizons, tile = _host(batch, i), _tile(patch)
        expected = products.psr_tile(dem, horizons, reduced, **tile)
        peak = products.psr_peak_margin(dem, horizons, reduced, **tile)
        band = np.abs(peak - products.PSR_LIMB_THRESHOLD) < 1e-4
        band_pixels += int(band.sum())
        assert not np.any((psr[i] != expected) & ~band), patch
    assert any(np.any(p == 255) for p in psr)
    assert band_pixels < 0.001 * sum(p.size for p in psr)


def test_chain_lighting_products_match_the_oracle(chain_case):
    """The chain's sun fractions, Earth-visibility fractions and Sun-only
    mission durations on its resident horizons against the CPU oracle fed the
    same horizons.

    Marched horizons are rough: next to an obstacle they change by degrees
    from one 0.25-deg bin to the next, so the few-ulp difference between
    CUDA's and glibc's atan2f in the Sun's azimuth moves the interpolated
    horizon, and with it the fraction, by up to ~1e-3 at such samples.  The
    1e-4 agreement holds for 99.9 % of the samples and every fraction is
    within 2e-3.  Visibility is exact except where a margin sits within
    1e-4 deg of the threshold, durations except at pixels where a fraction
    sits within 2e-3 of the 0.5 threshold."""
    from oracle import products

    chain, batch, dem = chain_case["chain"], chain_case["batch"], chain_case["dem"]
    sun, earth, hours = chain_case["sun"], chain_case["earth"], chain_case["hours"]
    fractions = chain.sun_fractions(batch, sun).cpu().numpy()
    visible = chain.earth_visibility(batch, earth)
    sample_hours = np.full(len(hours), 6.0)
    windows = np.array([[0, 40], [40, 100], [100, len(hours)]], dtype=np.int32)
    missions = chain.mission_durations(batch, sun, sample_hours=sample_hours,
                                       start_windows=windows)
    accepts = np.zeros((len(windows), len(hours)), dtype=bool)
    for i, (start, stop) in enumerate(windows):
        accepts[i, start:stop] = True
    for i, patch in enumerate(batch.patches[:2]):
        horizons, tile = _host(batch, i), _tile(patch)
        h, w = patch.height, patch.width
        expected = products.lighting_tiles(dem, horizons, sun, **tile)
        got = fractions[i].reshape(len(sun), 128, 128)[:, :h, :w]
        error = np.abs(got - expected)
        print(f"patch {i}: fraction error max {error.max():.2e}, "
              f"share within 1e-4 {np.mean(error <= 1e-4):.6f}")
        assert np.mean(error <= 1e-4) >= 0.999
        assert error.max() <= 2e-3
        margins = products.lighting_tiles(dem, horizons, earth, margin=True, **tile)
        near = np.any(np.abs(margins) < 1e-4, axis=0)
        expected_visible = products.earth_visibility(margins)
        assert not np.any((visible[i] != expected_visible) & ~near)
        expected_mission = products.longest_duration(expected >= np.float32(0.5),
                                                     sample_hours, accepts)
        edge = np.any(np.abs(expected - 0.5) < 2e-3, axis=0)
        assert not np.any((missions[i] != expected_mission) & ~edge[None])


def test_chain_validation(chain_case):
    from lunarscout_b200.chain import ProductChain

    chain = chain_case["chain"]
    with pytest.raises(ValueError):
        chain.march([])
    with pytest.raises(ValueError):
        chain.march(list(chain_case["patches"]) * 6)
    with pytest.raises(ValueError):
        ProductChain([chain_case["dem"]], traversal="sideways")
