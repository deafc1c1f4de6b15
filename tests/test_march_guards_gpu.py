"""Inputs on which a march could never end are refused before any launch.

The march (like the reference's kernel) advances its FP32 path position s
(km) by at least 1e-4 km per cull and half a pixel per level-0 sample.  When
an advance is below half an ulp of s, s stops moving and the ray steps in
place for ever.  The library refuses such inputs with ValueError: a DEM
whose pixel size is not positive, rays of 2048 km or more, and pixels too
small for the rays' length.  Nothing reaches the GPU in these tests.
"""

from __future__ import annotations

import numpy as np
import pytest

from conftest import pyramid_from

pytestmark = pytest.mark.gpu

COMMON = dict(tile_column=20, tile_row=20, tile_width=1, tile_height=1, subpatch_size=8)


def test_dem_with_zero_pixel_size_is_refused(cuda_session):
    class Dem:
        elevation_m = np.zeros((64, 64), dtype=np.float32)
        geo_transform = np.zeros(6)

        class projection:
            radius_m, latitude_origin_rad, longitude_origin_rad = 1737400.0, -1.5707963, 0.0
            scale, false_easting_m, false_northing_m = 1.0, 0.0, 0.0

    with np.errstate(divide="ignore"):
        device = cuda_session.upload_dem_grid(Dem)
    try:
        with pytest.raises(ValueError, match="pixel size"):
            cuda_session.generate_segments([device], tile_column=0, tile_row=0, tile_width=16,
                                           azimuth_count=8, maximum_distance_m=10_000.0,
                                           observer_elevation_m=0.0)
    finally:
        device.close()


def test_rays_of_2048_km_are_refused(production_case, cuda_session):
    arrays, pyramids = production_case
    segments = np.array(arrays["segments"], copy=True)
    segments[3, 1, 1, 13] = 2100.0  # one regional-pass ray ends beyond 2048 km
    with pytest.raises(ValueError, match="2048 km"):
        cuda_session.subpatch_hierarchical_all_passes(segments, pyramids, **COMMON)


def test_pixels_too_small_for_the_ray_length_are_refused(production_case, cuda_session):
    arrays, _ = production_case
    segments = np.array(arrays["segments"], copy=True)
    segments[..., 0, 13] = np.minimum(segments[..., 0, 13], 900.0)
    segments[0, 0, 0, 13] = 900.0
    tiny = dict(arrays)
    # A 3 mm pixel: half a pixel (1.5e-6 km) is below 2 ulp of 900 km.
    tiny["dem0_map"] = np.array(arrays["dem0_map"], copy=True)
    tiny["dem0_map"][6] = 3e-3
    tiny["dem0_map"][10] = -3e-3
    pyramid = pyramid_from(tiny, "dem0")
    with pytest.raises(ValueError, match="pixel size is too small"):
        cuda_session.subpatch_hierarchical_pass(segments, pyramid, pyramid, pass_index=0,
                                                **COMMON)


def test_segment_generation_refuses_rays_past_2048_km(cuda_session):
    from lunarscout_b200.synthetic import SyntheticDemSpec, synthetic_dem

    # 2000 px at 1 km: the ray limit (1.2 x the extent) is 2400 km.
    dem = synthetic_dem(SyntheticDemSpec(2000, 1000.0, sigma_m=500.0, craters=0, seed=4))
    device = cuda_session.upload_dem_grid(dem)
    try:
        with pytest.raises(ValueError, match="2048 km"):
            cuda_session.generate_segments([device], tile_column=896, tile_row=896,
                                           tile_width=128, azimuth_count=8,
                                           maximum_distance_m=3_000_000.0,
                                           observer_elevation_m=0.0)
        # Within 2048 km the same DEM is accepted.
        segments = cuda_session.generate_segments([device], tile_column=896, tile_row=896,
                                                  tile_width=128, azimuth_count=8,
                                                  maximum_distance_m=1_500_000.0,
                                                  observer_elevation_m=0.0)
        assert segments.shape == (8, (128 // 8 + 2) ** 2, 1, 18)
    finally:
        device.close()
