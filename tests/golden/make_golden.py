"""Generate the committed golden fixtures under tests/golden/.

Run with LUNARSCOUT_REFERENCE set to the root of a lunarscout source checkout
(read-only); the tests only read this script's outputs.  It imports the reference's own
Python modules through a stub package (its top-level ``__init__`` needs
pyproj/rasterio, absent here) and extracts:

* horizon_production.npz — the reference's single-pixel two-DEM production
  fixture (tests/data/numba_horizon/phase1_reference_rays.npz) with the
  segment tensor the reference's own tests feed it
  (geometry.build_subpatch_segments), the C# golden per-DEM and final slopes
  and the 932-row C# traversal trace (phase4d_production_segments.json), the
  C# bilinear-boundary trace, and the output of the reference's production
  Numba kernel (cuda_backend.subpatch_hierarchy_kernel) executed by Numba's
  CUDA simulator on CPU.
* pyramids.npz — C# pyramid captures incl. the NaN/inf/-20000 fixture.
* segments_halo.npz — the 16x16-tile, 16-azimuth, two-DEM halo fixture: the
  C# segment tensor, the reference's Numba segment tensor and its DEMs.
* safe_haven_reference.npz — the reference safe-haven reducer and month-band
  helpers on the reference CPU backend's lighting streams and on seeded
  synthetic streams (safe_haven_reference below).

Usage: LUNARSCOUT_REFERENCE=<checkout> python tests/golden/make_golden.py [--simulate]
(--simulate re-runs the simulator capture, ~5 min).
"""

from __future__ import annotations

import argparse
import json
import os
import sys
import types
from fractions import Fraction
from pathlib import Path

import numpy as np

if not os.environ.get("LUNARSCOUT_REFERENCE"):
    sys.exit("set LUNARSCOUT_REFERENCE to the root of a lunarscout source checkout")
REFERENCE_ROOT = Path(os.environ["LUNARSCOUT_REFERENCE"])
PACKAGE = REFERENCE_ROOT / "src" / "lunarscout"
DATA = REFERENCE_ROOT / "tests" / "data" / "numba_horizon"
OUT = Path(__file__).resolve().parent


def import_reference():
    os.environ.setdefault("NUMBA_CACHE_DIR", "/tmp/lunarscout-numba-cache")
    sys.dont_write_bytecode = True
    if "lunarscout" not in sys.modules:
        stub = types.ModuleType("lunarscout")
        stub.__path__ = [str(PACKAGE)]
        sys.modules["lunarscout"] = stub


def _artifact():
    from lunarscout._numba_horizon.contract import load_reference_artifact

    return load_reference_artifact(DATA / "phase1_reference_rays.json",
                                   DATA / "phase1_reference_rays.npz")


def _dem(artifact, prefix):
    from lunarscout._numba_horizon.geometry import DemGrid, ProjectionParameters

    return DemGrid(
        artifact.arrays[f"{prefix}__elevation_m"],
        artifact.arrays[f"{prefix}__geo_transform"],
        ProjectionParameters.from_array(artifact.arrays[f"{prefix}__pyramid__projection_parameters"]),
    )


def _pyramid_dict(artifact, prefix, name):
    from lunarscout._numba_horizon.contract import PyramidArrays

    p = PyramidArrays.from_artifact(artifact.arrays, f"{prefix}__pyramid")
    return {
        f"{name}_level0": p.level0,
        f"{name}_mips": p.mips,
        f"{name}_levels": p.levels,
        f"{name}_map": p.map_parameters,
        f"{name}_projection": p.projection_parameters,
    }


TRACE_FIELDS = ("s_km", "true_distance_m", "level", "cell_x", "cell_y", "pixel_x",
                "pixel_y", "maximum_elevation_m", "sample_elevation_m", "sample_slope",
                "advance_km", "action")


def _trace(capture):
    return np.asarray([[np.nan if row[f] is None else row[f] for f in TRACE_FIELDS]
                       for row in capture["trace"]], dtype=np.float32)


def _exact_fmaf(a, b, c):
    """Correctly rounded float32 fma (Numba's simulator has no libdevice)."""
    a, b, c = np.float32(a), np.float32(b), np.float32(c)
    exact = Fraction(float(a)) * Fraction(float(b)) + Fraction(float(c))
    r = np.float32(float(exact))
    best = None
    for cand in (np.nextafter(r, np.float32(-np.inf)), r, np.nextafter(r, np.float32(np.inf))):
        if not np.isfinite(cand):
            continue
        d = abs(Fraction(float(cand)) - exact)
        if best is None or d < best[0] or (d == best[0] and int(cand.view(np.uint32)) & 1 == 0):
            best = (d, cand)
    return best[1]


def simulate_reference_kernel(segments, pyramids):
    """Run the reference's production kernel under Numba's CUDA simulator."""
    os.environ["NUMBA_ENABLE_CUDASIM"] = "1"
    from types import SimpleNamespace

    import numba
    import numba.cuda.libdevice as libdevice
    from numba import cuda
    from numba.cuda.simulator import kernel as simkernel

    libdevice.fmaf = _exact_fmaf

    class CudaProxy:
        """Resolve cuda.* inside simulated kernels through the kernel context
        (the reference binds ``cuda`` as a closure, not a global)."""

        def __getattr__(self, name):
            context = simkernel._get_kernel_context()
            if context is not None and hasattr(context, name):
                return getattr(context, name)
            return getattr(cuda, name)

    original_jit = cuda.jit

    def jit(*args, **kwargs):
        kwargs.pop("max_registers", None)
        kwargs.pop("cache", None)
        return original_jit(*args, **kwargs)

    cuda.jit = jit
    cuda.get_current_device = lambda: SimpleNamespace(name=b"simulator",
                                                      compute_capability=(0, 0))
    import lunarscout._cuda_runtime as runtime

    runtime.import_numba_cuda = lambda: (numba, CudaProxy())
    from lunarscout._numba_horizon.cuda_backend import CudaSession

    session = CudaSession()
    common = dict(tile_column=20, tile_row=20, tile_width=1, tile_height=1, subpatch_size=8)
    pass0 = session.subpatch_hierarchical_pass(segments, pyramids[0], pyramids[0],
                                               pass_index=0, **common)
    final = session.subpatch_hierarchical_pass(segments, pyramids[0], pyramids[1],
                                               pass_index=1, slopes=pass0, **common)
    return pass0.reshape(-1), final.reshape(-1)


def horizon_production(simulate: bool) -> None:
    from lunarscout._numba_horizon.geometry import (
        GridConvergenceInput, build_subpatch_segments)
    from lunarscout._numba_horizon.contract import PyramidArrays

    artifact = _artifact()
    base = "single_pixel_multi_dem_production__horizon_buffer_fixture"
    dems = [_dem(artifact, f"{base}__dem_{i}") for i in range(2)]
    pyramids = [PyramidArrays.from_artifact(artifact.arrays, f"{base}__dem_{i}__pyramid")
                for i in range(2)]
    segments, _, _ = build_subpatch_segments(
        dems, tile_column=20, tile_row=20, tile_width=1, azimuth_count=1440,
        maximum_distance_m=1_000_000, observer_elevation_m=0, subpatch_size=8,
        grid_convergence=GridConvergenceInput(0.0, 0.0, 0.0))
    capture = json.loads((DATA / "phase4d_production_segments.json").read_text())
    production = capture["production_hierarchy_case"]
    boundary = capture["bilinear_boundary_case"]
    arrays = {
        "segments": segments.astype(np.float32),
        "csharp_per_dem_slopes": np.asarray(production["per_dem_slopes"], np.float32).reshape(2, 1440),
        "csharp_final_slopes": np.asarray(production["final_slopes"], np.float32),
        "csharp_final_degrees": np.asarray(production["final_degrees"], np.float32),
        "csharp_trace": _trace(production),
        "csharp_trace_segments": np.asarray(capture["segments"], np.float32),
        "csharp_trace_observer_z": np.float32(dems[0].elevation(20, 20)),
        "csharp_trace_maximum_slope": np.float32(production["csharp_hierarchy_maximum_slope"]),
        "boundary_segments": np.asarray(boundary["segments"], np.float32),
        "boundary_trace": _trace(boundary),
        "boundary_maximum_slope": np.float32(boundary["csharp_hierarchy_maximum_slope"]),
    }
    for i in range(2):
        arrays[f"dem{i}_geo_transform"] = dems[i].geo_transform
        arrays.update(_pyramid_dict(artifact, f"{base}__dem_{i}", f"dem{i}"))
    # The boundary case DEM (single_obstacle_north), its observer and resolution.
    case = next(c for c in artifact.metadata["cases"] if c["id"] == "single_obstacle_north")
    bdem = _dem(artifact, "single_obstacle_north__dem_0")
    arrays["boundary_elevation"] = bdem.elevation_m
    observer = case["observer"]
    arrays["boundary_observer_z"] = np.float32(
        float(bdem.elevation(observer["pixel_x"], observer["pixel_y"])) + float(observer["elevation_m"]))
    arrays["boundary_radius"] = np.float32(bdem.projection.radius_m)
    arrays["boundary_resolution"] = np.float32(case["ray_fit_passes"][0]["map_resolution_m"])
    target = OUT / "horizon_production.npz"
    if simulate or not target.exists():
        pass0, final = simulate_reference_kernel(segments, pyramids)
    else:
        with np.load(target) as old:
            pass0, final = old["reference_sim_pass0"], old["reference_sim_final"]
    arrays["reference_sim_pass0"] = pass0
    arrays["reference_sim_final"] = final
    np.savez_compressed(target, **arrays)


def pyramids_fixture() -> None:
    artifact = _artifact()
    arrays = {}
    names = []
    for case in artifact.metadata["cases"]:
        for pyramid in case["pyramids"]:
            prefix = f"{case['id']}__dem_{pyramid['dem_index']}__pyramid"
            levels = artifact.arrays[f"{prefix}__level_metadata"]
            if levels[0, 2] * levels[0, 3] > 5000:
                continue
            name = f"p{len(names)}"
            names.append(prefix)
            arrays[f"{name}_levels"] = levels
            for level in range(len(levels)):
                arrays[f"{name}_level{level}"] = artifact.arrays[f"{prefix}__level_{level}"]
    fixture = "invalid_values_odd_dimensions__pyramid_fixture"
    arrays["invalid_elevation"] = artifact.arrays[f"{fixture}__elevation_m"]
    arrays["invalid_levels"] = artifact.arrays[f"{fixture}__level_metadata"]
    for level in range(3):
        arrays[f"invalid_level{level}"] = artifact.arrays[f"{fixture}__level_{level}"]
    arrays["names"] = np.array(names)
    np.savez_compressed(OUT / "pyramids.npz", **arrays)


def segments_halo() -> None:
    from lunarscout._numba_horizon.geometry import (
        GridConvergenceInput, build_subpatch_segments_numba)

    artifact = _artifact()
    fixture = next(f for f in artifact.metadata["subpatch_fixtures"]
                   if f["id"] == "boundary_halo_multi_dem_16az")
    config = fixture["configuration"]
    dems = [_dem(artifact, f"multi_dem_outer_obstacle_east__dem_{i}") for i in range(2)]
    kwargs = dict(tile_column=config["tile_column"], tile_row=config["tile_row"],
                  tile_width=config["tile_width"], azimuth_count=config["azimuth_count"],
                  maximum_distance_m=config["max_distance_m"],
                  observer_elevation_m=config["observer_elevation_m"],
                  subpatch_size=config["subpatch_size"])
    numba_segments, _, _ = build_subpatch_segments_numba(
        dems, grid_convergence=GridConvergenceInput(0.0, 0.0, 0.0), parallel=False, **kwargs)
    arrays = {
        "csharp_segments": artifact.arrays["boundary_halo_multi_dem_16az__subpatch_fixture__segment_values"],
        "reference_numba_segments": numba_segments,
        "config": np.array([config["tile_column"], config["tile_row"], config["tile_width"],
                            config["tile_height"], config["subpatch_size"],
                            config["azimuth_count"], config["max_distance_m"]], dtype=np.int64),
    }
    for i, dem in enumerate(dems):
        arrays[f"dem{i}_elevation"] = dem.elevation_m
        arrays[f"dem{i}_geo_transform"] = dem.geo_transform
        arrays[f"dem{i}_projection"] = np.array(
            (dem.projection.radius_m, dem.projection.latitude_origin_rad,
             dem.projection.longitude_origin_rad, dem.projection.scale,
             dem.projection.false_easting_m, dem.projection.false_northing_m), np.float64)
    np.savez_compressed(OUT / "segments_halo.npz", **arrays)


def lighting_csharp() -> None:
    """C# BuilderSunFraction samples and ILGPU PSR tiles."""
    import base64

    lightmap = json.loads((DATA / "phase6b_lightmap_csharp.json").read_text())
    arrays = {}
    for index, case in enumerate(lightmap["cases"]):
        arrays[f"lm{index}_horizon"] = np.frombuffer(
            base64.b64decode(case["horizons_float32_base64"]), dtype="<f4").astype(np.float32)
        arrays[f"lm{index}_samples"] = np.array(
            [[s["azimuth_deg"], s["elevation_deg"], s["encoded_byte"], s["fraction_float32_bits"]]
             for s in case["samples"]], dtype=np.float64)
    psr = json.loads((DATA / "phase6b_psr_csharp.json").read_text())
    p = psr["projection"]
    arrays["psr_geo_transform"] = np.asarray(psr["geotransform"], dtype=np.float64)
    arrays["psr_projection"] = np.array(
        (p["radius_m"], p["latitude_origin_rad"], p["longitude_origin_rad"], p["scale"],
         p["false_easting_m"], p["false_northing_m"]), dtype=np.float64)
    names = []
    for index, case in enumerate(psr["cases"]):
        names.append(case["name"])
        arrays[f"psr{index}_vectors"] = np.asarray(case["sun_vectors_m"], np.float64).reshape(-1, 3)
        arrays[f"psr{index}_expected"] = np.frombuffer(
            base64.b64decode(case["output_base64"]), dtype=np.uint8).reshape(128, 128)
    arrays["psr_names"] = np.array(names)
    np.savez_compressed(OUT / "lighting_csharp.npz", **arrays)


def synthetic_horizons(height=128, width=128):
    """Deterministic horizon tile (degrees): smooth ridges in azimuth whose
    phase and level vary per pixel (the level rises across the tile, so that
    some pixels are permanently shadowed)."""
    az = np.radians(np.arange(1440, dtype=np.float64) * 0.25)
    y, x = np.mgrid[0:height, 0:width]
    phase = (0.05 * x + 0.03 * y)[..., None]
    level = (1.0 + 0.25 * (x - y))[..., None]
    h = level + 2.5 * np.sin(3.0 * az + phase) + 1.0 * np.sin(11.0 * az + 2.0 * phase)
    return np.ascontiguousarray(h, dtype=np.float32)


def lighting_reference() -> None:
    """Reference CPU backend outputs on the synthetic 512x512 site DEM."""
    sys.path.insert(0, str(OUT.parents[1]))
    from lunarscout._numba_horizon.lightmap_cpu import LightmapCpuSession
    from lunarscout._numba_horizon.mission_duration import (
        reduce_longest_candidate_duration_stream, weekly_candidate_intervals)
    from lunarscout._numba_horizon.psr import (
        compute_psr_patch_reference, reduce_sun_vectors_for_psr)
    from lunarscout_b200 import synthetic

    from lunarscout._numba_horizon.geometry import DemGrid, ProjectionParameters

    ours = synthetic.config1_dem()
    dem = DemGrid(ours.elevation_m, ours.geo_transform,
                  ProjectionParameters.from_array(ours.projection.as_array()))
    tile = dict(tile_y=448, tile_x=448, valid_height=40, valid_width=48)
    horizons = np.zeros((128, 128, 1440), dtype=np.float32)
    horizons[:] = synthetic_horizons()
    hours = synthetic.hours_between("2029-01-01T00", "2029-02-01T00", 6.0)
    sun = synthetic.sun_vectors(hours)
    earth = synthetic.earth_vectors(hours)
    session = LightmapCpuSession(time_batch_size=32)
    fractions = np.stack(list(session.iter_patch_fraction_tiles(dem, horizons, sun, **tile)))
    margins = np.stack(list(session.iter_patch_margin_tiles(dem, horizons, earth, **tile)))
    reduced, indices = reduce_sun_vectors_for_psr(dem, sun)
    psr = compute_psr_patch_reference(dem, horizons, reduced, **tile)
    psr_all = compute_psr_patch_reference(dem, horizons, sun, **tile)
    times = [f"2029-01-01T00:00:00+00:00"] * 0
    import datetime as dt

    start = dt.datetime(2029, 1, 1, tzinfo=dt.timezone.utc)
    times = [start + dt.timedelta(hours=float(h)) for h in hours]
    stop = start + dt.timedelta(days=31, hours=6)
    intervals = weekly_candidate_intervals(start, stop)
    durations = reduce_longest_candidate_duration_stream(
        (f >= np.float32(0.5) for f in fractions), times_utc=times, evaluation_start_utc=start,
        evaluation_stop_utc=stop, start_intervals=intervals, output_unit="hours")
    both = reduce_longest_candidate_duration_stream(
        ((f >= np.float32(0.5)) & (m >= np.float32(0.0)) for f, m in zip(fractions, margins)),
        times_utc=times, evaluation_start_utc=start, evaluation_stop_utc=stop,
        start_intervals=intervals, output_unit="days")
    np.savez_compressed(
        OUT / "lighting_reference.npz",
        tile=np.array([tile["tile_y"], tile["tile_x"], tile["valid_height"], tile["valid_width"]]),
        hours=hours, fractions=fractions.astype(np.float32), margins=margins.astype(np.float32),
        psr_reduced_indices=indices, psr_reduced=psr, psr_all=psr_all,
        durations_hours=np.stack(durations), durations_days_sun_earth=np.stack(both),
        interval_bounds_hours=np.array(
            [[(i.start_utc - start).total_seconds() / 3600.0,
              (i.stop_utc - start).total_seconds() / 3600.0] for i in intervals]),
        evaluation_stop_hours=np.float64((stop - start).total_seconds() / 3600.0),
    )


def safe_haven_reference() -> None:
    """The reference safe-haven reducer and its month-band helpers on (a) the
    reference CPU backend's fraction / Earth-margin tiles of
    lighting_reference.npz and (b) seeded synthetic streams over four months,
    with a second mapping whose first month is left out (-1) and whose times
    are not in order."""
    import datetime as dt

    from lunarscout._numba_horizon.safe_haven import (
        _month_indices_map, build_month_bands, reduce_safe_haven_patch_stream)

    def run(fractions, margins, months, bands, sunlight, earth, hours):
        out = reduce_safe_haven_patch_stream(
            iter(fractions), iter(margins), len(fractions), bands, month_index_of=months,
            sunlight_threshold=sunlight, earth_threshold_deg=earth, time_step_hours=hours)
        return np.stack(out)

    lighting = np.load(OUT / "lighting_reference.npz")
    start = dt.datetime(2029, 1, 1, tzinfo=dt.timezone.utc)
    times_a = [start + dt.timedelta(hours=float(h)) for h in lighting["hours"]]
    bands_a = build_month_bands(times_a)
    months_a = _month_indices_map(times_a, bands_a)
    fractions_a = lighting["fractions"]
    margins_a = lighting["margins"]
    sunlight_a = 0.5
    earth_a = float(np.median(margins_a))
    out_a = run(fractions_a, margins_a, months_a, bands_a, sunlight_a, earth_a, 6.0)

    rng = np.random.default_rng(20290120)
    count, height, width = 300, 12, 10
    first = dt.datetime(2029, 1, 20, 3, tzinfo=dt.timezone.utc)
    times_b = [first + dt.timedelta(hours=6 * i) for i in range(count)]
    low = np.zeros((count, height, width), dtype=bool)
    state = rng.random((height, width)) < 0.5
    for t in range(count):
        state ^= rng.random((height, width)) < 0.08
        low[t] = state
    fractions_b = np.where(low, rng.uniform(0.0, 0.19, low.shape),
                           rng.uniform(0.21, 1.0, low.shape)).astype(np.float32)
    walk = np.cumsum(rng.normal(0.0, 0.6, (count, height, width)), axis=0)
    margins_b = (2.0 + walk - walk.mean(axis=0)).astype(np.float32)
    margins_b[:, 0, :3] = 5.0        # never an outage: NaN
    margins_b[:, 1, :3] = -1.0       # always an outage: NaN
    margins_b[:, 2, 0] = np.float32(2.0)  # exactly at the threshold: not an outage
    fractions_b[:, 3, 0] = np.float32(0.2)  # exactly at the threshold: not low
    bands_b = build_month_bands(times_b)
    months_b = _month_indices_map(times_b, bands_b)
    out_b = run(fractions_b, margins_b, months_b, bands_b, 0.2, 2.0, 6.0)

    order = np.arange(count)
    order[40:60] = order[40:60][::-1]
    times_c = [times_b[i] for i in order]
    bands_c = bands_b[1:]
    months_c = _month_indices_map(times_c, bands_c)
    out_c = run(fractions_b, margins_b, months_c, bands_c, 0.2, 2.0, 1.5)

    iso = lambda values: np.array([v.isoformat() for v in values])
    np.savez_compressed(
        OUT / "safe_haven_reference.npz",
        a_months=months_a, a_bands=iso([b for band in bands_a for b in band]),
        a_sunlight=np.float64(sunlight_a), a_earth=np.float64(earth_a), a_out=out_a,
        b_times=iso(times_b), b_fractions=fractions_b, b_margins=margins_b, b_months=months_b,
        b_bands=iso([b for band in bands_b for b in band]), b_out=out_b,
        c_times=iso(times_c), c_months=months_c, c_out=out_c,
    )


def codec_reference() -> None:
    """The reference .cbin encoder on a deterministic degree tile."""
    import hashlib

    from lunarscout._numba_horizon.file_format import _decode_compressed_payload, _encode_horizons

    degrees = synthetic_horizons().reshape(-1, 1440) * np.float32(6.0)
    degrees[5, :7] = -np.inf          # sentinel pixels encode as -50
    degrees[9, 100:110] = 75.0        # clamps at +50
    encoded, lengths = _encode_horizons(np.ascontiguousarray(degrees, dtype=np.float32))
    payload = b"".join(int(n).to_bytes(2, "little") + encoded[i, :n].tobytes()
                       for i, n in enumerate(lengths))
    decoded = _decode_compressed_payload(np.frombuffer(payload, dtype=np.uint8))
    np.savez_compressed(
        OUT / "codec_reference.npz",
        payload_sha256=np.array(hashlib.sha256(payload).hexdigest()),
        payload_size=np.int64(len(payload)), lengths=lengths.astype(np.uint16),
        head=np.frombuffer(payload[:4096], dtype=np.uint8),
        decoded_rows=decoded[[0, 5, 9, 777, 16383]],
    )


def psr_reduction_reference() -> None:
    """The reference's reduce_sun_vectors_for_psr on long vector tables: one
    year hourly on the 512 x 512 synthetic site, and three years hourly on the
    4096 x 4096 site-scale DEM (only its five viewpoint elevations matter)."""
    sys.path.insert(0, str(OUT.parents[1]))
    from lunarscout._numba_horizon.geometry import DemGrid, ProjectionParameters
    from lunarscout._numba_horizon.psr import reduce_sun_vectors_for_psr
    from lunarscout_b200 import synthetic

    cases = {
        "plain_year": (synthetic.config1_dem(),
                       synthetic.hours_between("2030-01-01T00", "2031-01-01T00", 1.0)),
        "site_three_years": (synthetic.site_dem(),
                             synthetic.hours_between("2030-01-01T00", "2033-01-01T00", 1.0)),
    }
    arrays = {}
    for name, (ours, hours) in cases.items():
        dem = DemGrid(ours.elevation_m, ours.geo_transform,
                      ProjectionParameters.from_array(ours.projection.as_array()))
        _, indices = reduce_sun_vectors_for_psr(dem, synthetic.sun_vectors(hours))
        arrays[f"{name}_hours"] = np.array([hours[0], hours[-1], hours[1] - hours[0]])
        arrays[f"{name}_indices"] = indices.astype(np.int64)
    np.savez_compressed(OUT / "psr_reduction_reference.npz", **arrays)


def main() -> None:
    parser = argparse.ArgumentParser()
    parser.add_argument("--simulate", action="store_true")
    parser.add_argument("--only", default="")
    args = parser.parse_args()
    import_reference()
    jobs = {
        "horizon": lambda: horizon_production(args.simulate),
        "pyramids": pyramids_fixture,
        "segments": segments_halo,
        "lighting_csharp": lighting_csharp,
        "lighting_reference": lighting_reference,
        "codec": codec_reference,
        "safe_haven": safe_haven_reference,
        "psr_reduction": psr_reduction_reference,
    }
    for name, job in jobs.items():
        if args.only and name not in args.only.split(","):
            continue
        job()
        print("wrote", name)


if __name__ == "__main__":
    main()
