"""The persistent multi-site march on the B200: the reference traversal equals
the per-tile path bit for bit, the skip ladder equals its CPU restatement bit
for bit, on one batch mixing sites of different sizes, resolutions, DEM
counts and partial edge tiles."""

from __future__ import annotations

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

AZ = 48
DISTANCE = 60_000.0


@pytest.fixture(scope="module")
def site_dems():
    from lunarscout_b200.synthetic import SyntheticDemSpec, synthetic_dem

    site_a = synthetic_dem(SyntheticDemSpec(320, 20.0, latitude_deg=-88.5, longitude_deg=30.0,
                                            craters=30, seed=5))
    site_b = synthetic_dem(SyntheticDemSpec(200, 10.0, latitude_deg=-87.0, longitude_deg=120.0,
                                            craters=10, crater_max_m=800.0, seed=7))
    regional = synthetic_dem(SyntheticDemSpec(800, 240.0, latitude_deg=-90.0, sigma_m=1200.0,
                                              craters=0, tilt_m=2000.0, seed=1005))
    return site_a, site_b, regional


@pytest.fixture(scope="module")
def batch(site_dems, cuda_session):
    from lunarscout_b200.cuda_backend import SiteTile

    site_a, site_b, regional = site_dems
    a, b, r = (cuda_session.upload_dem_grid(d) for d in (site_a, site_b, regional))
    grids = {id(a): site_a, id(b): site_b, id(r): regional}
    tiles = [
        SiteTile((a, r), 0, 0, DISTANCE, 1.5),
        SiteTile((b,), 128, 0, DISTANCE, 0.0),          # partial, one DEM
        SiteTile((a, r), 256, 256, DISTANCE, 0.0),      # partial corner
        SiteTile((b, r), 0, 128, DISTANCE, 3.0),        # partial bottom
        SiteTile((a, r), 128, 128, DISTANCE, 0.0),
    ]
    return tiles, grids


def _run(session, tiles, traversal, degrees=False):
    import torch

    out = torch.empty(len(tiles) * 16384 * AZ, dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    seconds = session.march_sites(tiles, device_out=out.data_ptr(), azimuth_count=AZ,
                                  traversal=traversal, degrees=degrees)
    assert all(s >= 0.0 for s in seconds)
    return out.cpu().numpy().reshape(len(tiles), 16384, AZ)


def _per_tile(session, tile):
    import torch

    count = 128 // 8 + 2
    dems = list(tile.dems)
    segments = torch.empty(AZ * count * count * len(dems) * 18, dtype=torch.float32,
                           device="cuda")
    out = torch.empty(16384 * AZ, dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    session.generate_segments_device(dems, segments.data_ptr(), tile_column=tile.tile_column,
                                     tile_row=tile.tile_row, azimuth_count=AZ,
                                     maximum_distance_m=tile.maximum_distance_m,
                                     observer_elevation_m=tile.observer_elevation_m)
    session.march_all_passes_device(segments.data_ptr(), AZ, count * count, dems,
                                    tile_column=tile.tile_column, tile_row=tile.tile_row,
                                    observer_elevation_m=tile.observer_elevation_m,
                                    device_out=out.data_ptr())
    # The device entry points are asynchronous on the session's stream.
    session.synchronize()
    return out.cpu().numpy().reshape(16384, AZ)


def test_exact_traversal_equals_the_per_tile_path(batch, cuda_session):
    tiles, _ = batch
    got = _run(cuda_session, tiles, "exact")
    for t, tile in enumerate(tiles):
        np.testing.assert_array_equal(got[t], _per_tile(cuda_session, tile), err_msg=f"tile {t}")
    assert np.isfinite(got[0]).all()
    assert np.isneginf(got[1].reshape(128, 128, AZ)[:, 72:]).all()   # x >= 200 on site b


# The batched traversals and the oracle masks that restate them.
CPU_MASKS = {
    "ladder": oracle.ladder_mask(0, 1),
    "relative": oracle.PRODUCTION_MASK | oracle.OPT_RELATIVE,
    "relative-ladder": oracle.ladder_mask(0, 1) | oracle.OPT_RELATIVE,
}


@pytest.mark.parametrize("traversal", sorted(CPU_MASKS))
def test_batched_traversal_equals_its_cpu_restatement(batch, cuda_session, traversal):
    from lunarscout_b200.contract import PyramidArrays, map_parameters, projection_parameters

    tiles, grids = batch
    got = _run(cuda_session, tiles, traversal)
    for t, tile in enumerate(tiles):
        dems = [grids[id(d)] for d in tile.dems]
        segments = cuda_session.generate_segments(
            list(tile.dems), tile_column=tile.tile_column, tile_row=tile.tile_row,
            tile_width=128, azimuth_count=AZ, maximum_distance_m=tile.maximum_distance_m,
            observer_elevation_m=tile.observer_elevation_m, subpatch_size=8)
        pyramids = []
        for dem in dems:
            mips, levels = oracle.build_pyramid(dem.elevation_m)
            pyramids.append(PyramidArrays(dem.elevation_m, mips, levels, map_parameters(dem),
                                          projection_parameters(dem)))
        expected, _ = oracle.march_all_passes(
            segments, pyramids, tile_column=tile.tile_column, tile_row=tile.tile_row,
            observer_elevation_m=tile.observer_elevation_m, mask=CPU_MASKS[traversal])
        np.testing.assert_array_equal(got[t], expected, err_msg=f"tile {t}")


def test_degrees_output_and_ladder_distance_from_the_exact_traversal(batch, cuda_session):
    tiles, _ = batch
    exact = _run(cuda_session, tiles, "exact")
    ladder_degrees = _run(cuda_session, tiles, "ladder", degrees=True)
    ladder = _run(cuda_session, tiles, "ladder")
    np.testing.assert_array_equal(ladder_degrees,
                                  cuda_session.slopes_to_degrees(ladder.reshape(-1, AZ))
                                  .reshape(ladder.shape))
    exact_degrees = cuda_session.slopes_to_degrees(exact.reshape(-1, AZ)).reshape(exact.shape)
    finite = np.isfinite(exact_degrees)
    assert np.array_equal(finite, np.isfinite(ladder_degrees))
    error = np.abs(ladder_degrees[finite].astype(np.float64) - exact_degrees[finite])
    assert np.quantile(error, 0.999) < 0.01, float(np.quantile(error, 0.999))


def test_ladder_visits_fewer_nodes(batch, cuda_session):
    tiles, _ = batch
    cuda_session.set_counting(True)
    try:
        _run(cuda_session, tiles, "exact")
        exact = cuda_session.last_counters()
        _run(cuda_session, tiles, "ladder")
        ladder = cuda_session.last_counters()
    finally:
        cuda_session.set_counting(False)
    assert ladder[2] < exact[2]          # ray steps
    assert ladder[0] < exact[0]          # node visits


def test_batch_validation(batch, cuda_session):
    import torch

    from lunarscout_b200.cuda_backend import SiteTile

    tiles, _ = batch
    out = torch.empty(16384 * AZ, dtype=torch.float32, device="cuda")
    with pytest.raises(ValueError):
        cuda_session.march_sites(tiles[:1], device_out=out.data_ptr(), azimuth_count=AZ,
                                 traversal="fast")
    with pytest.raises(ValueError):
        cuda_session.march_sites([SiteTile(tiles[0].dems * 5, 0, 0)], device_out=out.data_ptr(),
                                 azimuth_count=AZ)
    with pytest.raises(ValueError):
        cuda_session.march_sites([SiteTile(tiles[0].dems, 4096, 0)], device_out=out.data_ptr(),
                                 azimuth_count=AZ)
    with pytest.raises(ValueError):
        cuda_session.march_sites([], device_out=out.data_ptr(), azimuth_count=AZ)


@pytest.mark.parametrize("traversal", ["exact", "ladder", "relative-ladder"])
def test_results_are_invariant_across_launch_configurations(batch, cuda_session, traversal):
    from lunarscout_b200.autotune import DEFAULT_CANDIDATES

    tiles, _ = batch
    default = cuda_session.batch_config()
    reference = _run(cuda_session, tiles, traversal)
    try:
        for config in DEFAULT_CANDIDATES:
            cuda_session.set_batch_config(config)
            np.testing.assert_array_equal(_run(cuda_session, tiles, traversal), reference,
                                          err_msg=str(config))
    finally:
        cuda_session.set_batch_config(default)


def test_autotuner_times_every_candidate_and_applies_the_winner(batch, cuda_session):
    import torch

    from lunarscout_b200.autotune import DEFAULT_CANDIDATES, tune_batch
    from lunarscout_b200.cuda_backend import BatchConfig

    tiles, _ = batch
    default = cuda_session.batch_config()
    out = torch.empty(len(tiles) * 16384 * AZ, dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    try:
        result = tune_batch(cuda_session, tiles, device_out=out.data_ptr(), azimuth_count=AZ)
        assert set(result.seconds) == set(DEFAULT_CANDIDATES)
        assert all(s > 0.0 for s in result.seconds.values())
        assert cuda_session.batch_config() == result.best
    finally:
        cuda_session.set_batch_config(default)
    with pytest.raises(ValueError):
        cuda_session.set_batch_config(BatchConfig(12, 8))
    with pytest.raises(ValueError):
        cuda_session.set_batch_config(BatchConfig(32, 7))
    assert cuda_session.batch_config() == default
