"""Benchmark: the horizon march of the site-scale workload on B200.

One step = the production horizon march (both DEM passes, primary 4096x4096
at 5 m + regional 2000x2000 at 240 m, 200 km range) over one 128x128 tile with
1440 azimuths = 23,592,960 rays.  Tiles rotate every step (row-major tiles of
the primary DEM, rank r of N taking tiles r, r+N, ...: weak scaling, no data
collective).  Inputs are seeded synthetic DEMs (fBm + craters) with the
configuration's shapes; the per-step working set (segments 67 MB + DEM and
pyramids 106 MB + output 94 MB) exceeds the 126 MB L2.

value:  rays/s over all ranks with segments already resident in HBM (device
        march + transpose, CUDA events on the launch stream, max over ranks).
e2e:    rays/s through the drop-in CudaSession.subpatch_hierarchical_all_passes
        call with pinned host buffers (segments H2D + slopes D2H every step).
cpu_baseline: the oracle's C restatement of the march (all host threads) on a
        bounded random sample of rays of the same tiles (rank 0, N=1 only).

--impl reference: the reference algorithm's CPU restatement (oracle port; the
reference has no CPU horizon path of its own) on the host cores, same metric.
"""

from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "horizon rays/s & lightmap px·steps/s, 1 B200: batched vs plain, adjoint/fwd"
TILE = 128
AZIMUTHS = 1440
RAYS_PER_TILE = TILE * TILE * AZIMUTHS
RANGE_M = 200_000.0
OBSERVER_M = 0.0
# Algorithmic FP32 flops (FMA = 2) per unit of the march, counted from the
# reference source (cuda_backend.py:672-867): per ray step (two quartics,
# planar distance, chord cubic, footprint, level choice, two tangents and
# their reciprocals), per node visit (slab exit, fallback, near distance,
# four-cell local-z bound, step) and per level-0 sample (bilinear, local-z
# slope, tangent norm and the adaptive step rule).
FLOPS_PER_STEP = 67
FLOPS_PER_VISIT = 31
FLOPS_PER_SAMPLE = 35
# Bytes a node visit gathers (4 float32 cells) and a level-0 sample adds.
BYTES_PER_VISIT = 16
BYTES_PER_SAMPLE = 16


def log(*args):
    print(*args, file=sys.stderr, flush=True)


def profiled_traffic(name: str):
    """DRAM bytes per launch recorded by the committed ncu summary, if any."""
    path = ROOT / "profiles" / name
    try:
        for line in path.read_text().splitlines():
            if line.startswith("dram_bytes_per_launch:"):
                return int(line.split(":", 1)[1])
    except OSError:
        return None
    return None


def max_over_ranks(value: float, world: int, device: str = "cuda") -> float:
    """The maximum of a per-rank timing over all ranks (the job's time)."""
    if world <= 1:
        return value
    import torch
    import torch.distributed as dist

    t = torch.tensor([value], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def workload_config():
    return {
        "workload": "site-scale horizon march: 128x128 tile x 1440 az, 2 DEM passes",
        "primary_dem": "4096x4096 f32 @ 5 m, fBm sigma 150 m H 0.8 + 600 craters <= 8 km",
        "regional_dem": "2000x2000 f32 @ 240 m, fBm sigma 1.2 km + 2 km tilt",
        "range_km": RANGE_M / 1000.0,
        "azimuths": AZIMUTHS,
        "rays_per_step": RAYS_PER_TILE,
        "l2": "inputs larger than L2 (67 MB segments + 106 MB DEMs/pyramids + 94 MB "
              "output per step), tile changes every step",
    }


def tile_schedule(rank, world, count):
    tiles_per_side = 4096 // TILE
    # Start in the DEM interior so every step is a full tile with long rays.
    order = [(ty, tx) for ty in range(4, tiles_per_side - 4) for tx in range(4, tiles_per_side - 4)]
    rng = np.random.default_rng(1234)
    rng.shuffle(order)
    picked = [order[(rank + k * world) % len(order)] for k in range(count)]
    return [(ty * TILE, tx * TILE) for ty, tx in picked]


class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.device_index = device_index
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device_index}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.thread.join(timeout=2)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def build_dems():
    from lunarscout_b200.synthetic import regional_dem, site_dem

    started = time.perf_counter()
    primary = site_dem()
    regional = regional_dem()
    log(f"[bench] synthetic DEMs in {time.perf_counter() - started:.1f}s")
    return primary, regional


def cpu_sample_rate(primary, regional, tiles, seconds_target=12.0, threads=None):
    """Oracle march throughput (rays/s) on a bounded random ray sample."""
    import oracle
    from oracle import segments as oseg
    from lunarscout_b200.contract import PyramidArrays, map_parameters, projection_parameters

    pyramids = []
    for dem in (primary, regional):
        mips, levels = oracle.build_pyramid(dem.elevation_m)
        pyramids.append(PyramidArrays(dem.elevation_m, mips, levels, map_parameters(dem),
                                      projection_parameters(dem)))
    threads = threads or oracle.default_threads()
    tile_row, tile_column = tiles[0]
    segments = oseg.build_segments([primary, regional], tile_column=tile_column,
                                   tile_row=tile_row, tile_width=TILE, azimuth_count=AZIMUTHS,
                                   maximum_distance_m=RANGE_M, observer_elevation_m=OBSERVER_M,
                                   threads=threads)
    rng = np.random.default_rng(7)
    count = 256
    elapsed = 0.0
    rays = 0
    while elapsed < seconds_target:
        pixels = rng.integers(0, TILE * TILE, size=count).astype(np.int32)
        azimuths = rng.integers(0, AZIMUTHS, size=count).astype(np.int32)
        started = time.perf_counter()
        oracle.march_all_passes(segments, pyramids, tile_column=tile_column, tile_row=tile_row,
                                observer_elevation_m=OBSERVER_M, pixels=pixels,
                                azimuths=azimuths, threads=threads)
        took = time.perf_counter() - started
        elapsed += took
        rays += count
        if took < 1.0:
            count *= 4
    return rays / elapsed, threads, rays, elapsed


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    primary, regional = build_dems()
    tiles = tile_schedule(0, 1, 1)
    per_step = []
    rates = []
    for step in range(args.warmup + args.steps):
        rate, threads, rays, elapsed = cpu_sample_rate(primary, regional, tiles,
                                                       seconds_target=args.reference_seconds)
        if step >= args.warmup:
            rates.append(rate)
            per_step.append(elapsed)
    value = statistics.median(rates)
    line = {
        "impl": "reference",
        "metric": METRIC, "value": value, "unit": "rays/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000.0 * RAYS_PER_TILE / value,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": workload_config(),
        "cpu_baseline": {"value": value, "unit": "rays/s", "cores": threads, "kind": "port",
                         "sample": f"random rays of a site-scale tile, both DEM passes, "
                                   f"~{args.reference_seconds:.0f} s of CPU work per step"},
        "e2e": {"value": value, "unit": "rays/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


LIGHT_TILES = 8
# Per pixel x time step of the sun-fraction lightmap (lightmap_cpu.py:105-183):
# rotate (9 mul + 9 add), radicand + sqrt, 2 atan2, 3 mul/add to degrees, bin
# selection (6) and 16 slices of (fma-free lerp 2, add, compare/clamp 3, add,
# fraction step 2) = about 150 FP32 operations; 1 byte written.
LIGHT_FLOPS_PER_SAMPLE = 150


def safe_haven_benchmark(session, lib, count, patches, geo, proj, windows, horizons, world):
    """The fused safe-haven product (Sun fraction and Earth margin per pixel
    and step, then the per-month run reducer) over two years of hourly Sun
    and Earth vectors (17,545 steps, 25 month bands) on the same tiles."""
    import ctypes
    from datetime import datetime, timedelta, timezone

    import torch

    from lunarscout_b200 import _native, synthetic
    from lunarscout_b200.lightmap_cuda import DeviceVectors
    from lunarscout_b200.safe_haven import month_bands, month_indices

    hours = synthetic.hours_between("2030-01-01T00", "2032-01-01T00", 1.0)
    start = datetime(2030, 1, 1, tzinfo=timezone.utc)
    times = [start + timedelta(hours=float(h)) for h in hours]
    bands = month_bands(times)
    months = month_indices(times, bands)
    sun = DeviceVectors(session.context, synthetic.sun_vectors(hours).astype(np.float32))
    earth = DeviceVectors(session.context, synthetic.earth_vectors(hours).astype(np.float32))
    out = torch.empty((count, len(bands), TILE * TILE), dtype=torch.float32, device="cuda")

    def launch():
        _native.check(lib.ls200_safe_haven_device(
            session.context, count, ctypes.c_void_p(patches.data_ptr()), geo.ctypes.data,
            proj.ctypes.data, windows.ctypes.data, ctypes.c_void_p(horizons.data_ptr()),
            sun.handle, earth.handle, ctypes.c_float(0.2), ctypes.c_float(2.0),
            ctypes.c_float(1.0), months.ctypes.data, len(bands),
            ctypes.c_void_p(out.data_ptr())))

    launch()
    torch.cuda.synchronize()
    repeats = 3
    begin, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    begin.record()
    for _ in range(repeats):
        launch()
    end.record()
    torch.cuda.synchronize()
    elapsed = max_over_ranks(begin.elapsed_time(end) / 1000.0, world)
    sun.close()
    earth.close()
    px_steps = repeats * count * TILE * TILE * len(hours)
    finite = torch.isfinite(out)
    return {
        "metric": "safe-haven px·steps/s (Sun fraction + Earth margin + monthly run reducer)",
        "value": world * px_steps / elapsed, "unit": "px·steps/s", "tiles_per_launch": count,
        "time_steps": len(hours), "month_bands": len(bands), "launches": repeats,
        "ms_per_tile_two_years": 1000.0 * elapsed / (repeats * count),
        "defined_fraction": float(finite.float().mean()),
    }


def lighting_benchmark(session, dems, segments, tiles, primary, args, world, rank):
    """Sun-fraction bytes for one year of hourly steps on the timed tiles'
    horizons, computed from the device-resident march output (horizon ->
    degrees -> lightmap on the device, no host round trip)."""
    import ctypes

    import torch
    import torch.distributed as dist

    from lunarscout_b200 import _native, synthetic
    from lunarscout_b200.contract import projection_array
    from lunarscout_b200.lightmap_cuda import DeviceVectors

    count = min(LIGHT_TILES, args.steps)
    picks = list(range(args.warmup, args.warmup + count))
    plane = TILE * TILE
    horizons = torch.empty((count, plane, AZIMUTHS), dtype=torch.float32, device="cuda")
    patches = torch.empty((count, TILE, TILE), dtype=torch.float32, device="cuda")
    windows = np.zeros((count, 4), dtype=np.int32)
    elevation = torch.from_numpy(primary.elevation_m).to("cuda")
    centers = (TILE // 8 + 2) ** 2
    for i, k in enumerate(picks):
        tile_row, tile_column = tiles[k]
        session.march_all_passes_device(segments[k].data_ptr(), AZIMUTHS, centers, dems,
                                        tile_column=tile_column, tile_row=tile_row,
                                        observer_elevation_m=OBSERVER_M,
                                        device_out=horizons[i].data_ptr(), degrees=True)
        patches[i] = elevation[tile_row:tile_row + TILE, tile_column:tile_column + TILE]
        windows[i] = (tile_column, tile_row, TILE, TILE)
    torch.cuda.synchronize()
    geo = np.ascontiguousarray(np.repeat(primary.geo_transform[None, :], count, 0))
    proj = np.ascontiguousarray(np.repeat(projection_array(primary.projection)[None, :],
                                          count, 0))
    hours = synthetic.hours_between("2030-01-01T00", "2031-01-01T00", 1.0)
    vectors = synthetic.sun_vectors(hours).astype(np.float32)
    table = DeviceVectors(session.context, vectors)
    steps = len(vectors)
    frames = torch.empty(count * plane * 12, dtype=torch.float32, device="cuda")
    out = torch.empty((count, steps, plane), dtype=torch.uint8, device="cuda")
    lib = _native.library()

    def launch():
        _native.check(lib.ls200_lighting_device(
            session.context, count, ctypes.c_void_p(patches.data_ptr()), geo.ctypes.data,
            proj.ctypes.data, windows.ctypes.data, ctypes.c_void_p(horizons.data_ptr()),
            table.handle, 0, steps, 1, ctypes.c_void_p(frames.data_ptr()),
            ctypes.c_void_p(out.data_ptr())))

    for _ in range(3):
        launch()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    repeats = 5
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record()
    for _ in range(repeats):
        launch()
    end.record()
    torch.cuda.synchronize()
    elapsed = max_over_ranks(start.elapsed_time(end) / 1000.0, world)
    samples = repeats * count * plane * steps
    value = world * samples / elapsed
    table.close()
    haven = safe_haven_benchmark(session, lib, count, patches, geo, proj, windows, horizons,
                                 world)
    result = {
        "safe_haven": haven,
        "metric": "lightmap px·steps/s (sun-fraction bytes, 1 year hourly)",
        "value": value, "unit": "px·steps/s", "tiles_per_launch": count,
        "time_steps": steps, "launches": repeats,
        "ms_per_tile_year": 1000.0 * elapsed / (repeats * count),
        "achieved_tflops": value * LIGHT_FLOPS_PER_SAMPLE / 1e12,
        "output_gbs": value / 1e9,
    }
    if rank == 0 and world == 1 and not args.skip_cpu:
        import oracle  # noqa: F401  (CPU leg only)
        from oracle import products

        host_horizons = horizons[0].cpu().numpy().reshape(TILE, TILE, AZIMUTHS)
        tile_row, tile_column = tiles[picks[0]]
        sample = vectors.astype(np.float64)  # one tile, the whole year
        started = time.perf_counter()
        products.lighting_tiles(primary, host_horizons, sample, tile_y=tile_row,
                                tile_x=tile_column)
        took = time.perf_counter() - started
        result["cpu_baseline"] = {
            "value": plane * len(sample) / took, "unit": "px·steps/s",
            "cores": products.default_threads(), "kind": "port",
            "sample": f"one tile x {len(sample)} hourly steps ({took:.1f} s)"}
    return result


SITES = 64
SITE_TILES_PER_BATCH = 16
SITE_BATCHES = 3  # one warm-up batch, then timed batches
TUNE_TILES = 4
ACCURACY_RAYS_PER_TILE = 512


def multisite_benchmark(session, stream, args, world, rank):
    """The uneven multi-site workload (64 sites, sides 256-2048 px at 5-40 m,
    latitudes -83 to -89.5, one polar 240 m regional DEM, 200 km rays): each
    batch is one tile from each of 16 sites.  Plain = per-tile device segments
    + per-pass launches + transpose; batched = one persistent work-stealing
    launch over the whole batch (reference traversal, then skip ladder), its
    launch configuration chosen by the autotuner on part of the warm-up
    batch.  All produce degrees in HBM and are timed with CUDA events."""
    import torch
    import torch.distributed as dist

    from lunarscout_b200 import synthetic
    from lunarscout_b200.autotune import tune_batch
    from lunarscout_b200.cuda_backend import SiteTile

    started = time.perf_counter()
    specs = synthetic.multisite_specs(SITES)
    grids = [synthetic.synthetic_dem(spec) for spec in specs]
    regional = synthetic.polar_regional_dem()
    log(f"[bench] {SITES} site DEMs in {time.perf_counter() - started:.1f}s")
    regional_dev = session.upload_dem_grid(regional)
    site_devs = [session.upload_dem_grid(grid) for grid in grids]
    rng = np.random.default_rng(77 + rank)
    batches, picks = [], []
    for b in range(SITE_BATCHES):
        tiles, chosen = [], []
        for j in range(SITE_TILES_PER_BATCH):
            site = (rank * SITE_TILES_PER_BATCH * SITE_BATCHES + b * SITE_TILES_PER_BATCH + j) % SITES
            grid = grids[site]
            tx = int(rng.integers(0, (grid.width + TILE - 1) // TILE)) * TILE
            ty = int(rng.integers(0, (grid.height + TILE - 1) // TILE)) * TILE
            tiles.append(SiteTile((site_devs[site], regional_dev), tx, ty, RANGE_M, OBSERVER_M))
            chosen.append(site)
        batches.append(tiles)
        picks.append(chosen)
    timed_rays = sum(min(TILE, grids[s].width - t.tile_column)
                     * min(TILE, grids[s].height - t.tile_row) * AZIMUTHS
                     for tiles, chosen in zip(batches[1:], picks[1:])
                     for t, s in zip(tiles, chosen))
    centers = (TILE // 8 + 2) ** 2
    segments = torch.empty(AZIMUTHS * centers * 2 * 18, dtype=torch.float32, device="cuda")
    out = torch.empty((SITE_TILES_PER_BATCH, TILE * TILE, AZIMUTHS), dtype=torch.float32,
                      device="cuda")
    torch.cuda.synchronize()

    def plain(tiles):
        for i, tile in enumerate(tiles):
            dems = list(tile.dems)
            session.generate_segments_device(dems, segments.data_ptr(),
                                             tile_column=tile.tile_column,
                                             tile_row=tile.tile_row, azimuth_count=AZIMUTHS,
                                             maximum_distance_m=RANGE_M,
                                             observer_elevation_m=OBSERVER_M)
            session.march_all_passes_device(segments.data_ptr(), AZIMUTHS, centers, dems,
                                            tile_column=tile.tile_column,
                                            tile_row=tile.tile_row,
                                            observer_elevation_m=OBSERVER_M,
                                            device_out=out[i].data_ptr(), degrees=True)

    splits = {}  # traversal -> [(segment + setup seconds, march seconds)] per call

    def batched(traversal):
        def run(tiles):
            splits.setdefault(traversal, []).append(session.march_sites(
                tiles, device_out=out.data_ptr(), azimuth_count=AZIMUTHS, traversal=traversal,
                degrees=True))
        return run

    def timed(run):
        run(batches[0])
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record(stream)
        for tiles in batches[1:]:
            run(tiles)
        end.record(stream)
        torch.cuda.synchronize()
        elapsed = max_over_ranks(start.elapsed_time(end) / 1000.0, world)
        return world * timed_rays / elapsed, elapsed

    tuned = tune_batch(session, batches[0][:TUNE_TILES], device_out=out.data_ptr(),
                       azimuth_count=AZIMUTHS, traversal="ladder")
    plain_value, plain_s = timed(plain)
    exact_value, exact_s = timed(batched("exact"))
    ladder_value, ladder_s = timed(batched("ladder"))
    result = {
        "metric": "multi-site horizon rays/s (uneven batch, 2 DEM passes, 200 km)",
        "unit": "rays/s",
        "plain_per_tile": plain_value,
        "batched_exact": exact_value,
        "batched_ladder": ladder_value,
        "speedup_batched_vs_plain": ladder_value / plain_value,
        "speedup_exact_vs_plain": exact_value / plain_value,
        "seconds": {"plain": plain_s, "exact": exact_s, "ladder": ladder_s},
        "batched_split_seconds": {
            traversal: {"segments_and_setup": sum(s for s, _ in calls[-(SITE_BATCHES - 1):]),
                        "march": sum(m for _, m in calls[-(SITE_BATCHES - 1):])}
            for traversal, calls in splits.items()},
        "launch_config": {"lanes_per_azimuth": tuned.best.lanes_per_azimuth,
                          "min_blocks": tuned.best.min_blocks,
                          "tuned_on": f"{TUNE_TILES} tiles of the warm-up batch, ladder",
                          "candidates_ms": {
                              f"lanes{c.lanes_per_azimuth}/blocks{c.min_blocks}":
                                  1000.0 * s for c, s in tuned.seconds.items()}},
        "sites": SITES, "tiles_per_batch": SITE_TILES_PER_BATCH,
        "timed_batches": SITE_BATCHES - 1, "rays_timed_per_rank": timed_rays,
        "rays": "rays of pixels inside each site DEM (partial edge tiles count their valid part)",
    }
    result["pipeline"] = multisite_pipeline(session, stream, grids, batches[1], picks[1], out,
                                            plain, batched)
    if rank == 0 and world == 1 and not args.skip_cpu:
        result["error_vs_fp64_deg"] = multisite_accuracy(session, grids, regional, batches[1],
                                                         picks[1], out, batched)
    for dem in site_devs + [regional_dev]:
        dem.close()
    return result


PIPELINE_CHUNK = 1024


def multisite_pipeline(session, stream, grids, tiles, chosen, out, plain, batched):
    """Horizons + one year of hourly sun-fraction bytes + PSR for one batch
    of 16 site tiles.  Batched: the persistent ladder march, then the
    lightmap as a CUDA graph of 1024-step chunks over all tiles, then PSR.
    Plain: per tile, the per-tile march, the chunked lightmap and PSR
    launched eagerly.  Both keep results in HBM; CUDA events."""
    import ctypes

    import torch

    from lunarscout_b200 import _native, synthetic
    from lunarscout_b200.contract import projection_array
    from lunarscout_b200.graphs import DeviceGraph
    from lunarscout_b200.lightmap_cuda import DeviceVectors

    count = len(tiles)
    plane = TILE * TILE
    hours = synthetic.hours_between("2030-01-01T00", "2031-01-01T00", 1.0)
    vectors = synthetic.sun_vectors(hours).astype(np.float32)
    table = DeviceVectors(session.context, vectors)
    steps = len(vectors)
    patches = torch.zeros((count, TILE, TILE), dtype=torch.float32, device="cuda")
    geo = np.zeros((count, 6), dtype=np.float64)
    proj = np.zeros((count, 6), dtype=np.float64)
    windows = np.zeros((count, 4), dtype=np.int32)
    for i, (tile, site) in enumerate(zip(tiles, chosen)):
        grid = grids[site]
        vw = min(TILE, grid.width - tile.tile_column)
        vh = min(TILE, grid.height - tile.tile_row)
        patches[i, :vh, :vw] = torch.from_numpy(np.ascontiguousarray(
            grid.elevation_m[tile.tile_row:tile.tile_row + vh,
                             tile.tile_column:tile.tile_column + vw])).cuda()
        geo[i] = grid.geo_transform
        proj[i] = projection_array(grid.projection)
        windows[i] = (tile.tile_column, tile.tile_row, vw, vh)
    frames = torch.empty(count * plane * 12, dtype=torch.float32, device="cuda")
    chunk_out = torch.empty((count, PIPELINE_CHUNK, plane), dtype=torch.uint8, device="cuda")
    psr = torch.empty((count, plane), dtype=torch.uint8, device="cuda")
    lib = _native.library()
    blocks = [(start, min(PIPELINE_CHUNK, steps - start))
              for start in range(0, steps, PIPELINE_CHUNK)]
    torch.cuda.synchronize()

    def lighting(first, n, signal, target):
        _native.check(lib.ls200_lighting_device(
            session.context, n, ctypes.c_void_p(patches[first].data_ptr()),
            geo[first:].ctypes.data, proj[first:].ctypes.data, windows[first:].ctypes.data,
            ctypes.c_void_p(out[first].data_ptr()), table.handle, 0, steps, signal,
            ctypes.c_void_p(frames.data_ptr()), ctypes.c_void_p(target)))

    def lightmap_chunks(first, n):
        for start, length in blocks:
            _native.check(lib.ls200_lighting_device(
                session.context, n, ctypes.c_void_p(patches[first].data_ptr()),
                geo[first:].ctypes.data, proj[first:].ctypes.data, windows[first:].ctypes.data,
                ctypes.c_void_p(out[first].data_ptr()), table.handle, start, length, 1,
                ctypes.c_void_p(frames.data_ptr()), ctypes.c_void_p(chunk_out.data_ptr())))

    batched("ladder")(tiles)
    torch.cuda.synchronize()
    graph = DeviceGraph.capture(session.context, lambda: lightmap_chunks(0, count))

    def timed(run):
        run()
        torch.cuda.synchronize()
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record(stream)
        run()
        end.record(stream)
        torch.cuda.synchronize()
        return start.elapsed_time(end) / 1000.0

    def batched_pipeline():
        batched("ladder")(tiles)
        graph.launch()
        lighting(0, count, 3, psr.data_ptr())

    def plain_pipeline():
        plain(tiles)
        for i in range(count):
            lightmap_chunks(i, 1)
            lighting(i, 1, 3, psr[i].data_ptr())

    try:
        batched_s = timed(batched_pipeline)
        plain_s = timed(plain_pipeline)
        lightmap_graph_s = timed(graph.launch)
        graph_nodes = graph.nodes
    finally:
        graph.close()
        table.close()
    rays = sum(w[2] * w[3] for w in windows) * AZIMUTHS
    samples = sum(w[2] * w[3] for w in windows) * steps
    return {
        "tiles": count, "time_steps": steps, "chunk_steps": PIPELINE_CHUNK,
        "graph_nodes_per_batch": graph_nodes,
        "batched_seconds": batched_s, "plain_seconds": plain_s,
        "speedup_batched_vs_plain": plain_s / batched_s,
        "batched_rays_per_s": rays / batched_s,
        "lightmap_graph_px_steps_per_s": samples / lightmap_graph_s,
        "work": "ladder march (degrees) + sun-fraction bytes, 1 year hourly, in 1024-step "
                "graph-captured chunks + PSR over the same vectors",
    }


def multisite_accuracy(session, grids, regional, tiles, chosen, out, batched):
    """Horizon error of both traversals against the FP64 restatement of the
    reference march on a bounded ray sample of the first timed batch."""
    import oracle
    from lunarscout_b200.contract import PyramidArrays, map_parameters, projection_parameters

    def pyramid(dem):
        mips, levels = oracle.build_pyramid(dem.elevation_m)
        return PyramidArrays(dem.elevation_m, mips, levels, map_parameters(dem),
                             projection_parameters(dem))

    regional_pyramid = pyramid(regional)
    values = {}
    for traversal in ("exact", "ladder"):
        batched(traversal)(tiles)
        values[traversal] = out[:4].cpu().numpy()
    rng = np.random.default_rng(9)
    errors = {"exact": [], "ladder": []}
    for i, (tile, site) in enumerate(list(zip(tiles, chosen))[:4]):
        grid = grids[site]
        width = min(TILE, grid.width - tile.tile_column)
        height = min(TILE, grid.height - tile.tile_row)
        rows = rng.integers(0, height, ACCURACY_RAYS_PER_TILE)
        cols = rng.integers(0, width, ACCURACY_RAYS_PER_TILE)
        pixels = (rows * TILE + cols).astype(np.int32)
        azimuths = rng.integers(0, AZIMUTHS, ACCURACY_RAYS_PER_TILE).astype(np.int32)
        segments = session.generate_segments(list(tile.dems), tile_column=tile.tile_column,
                                             tile_row=tile.tile_row, azimuth_count=AZIMUTHS,
                                             maximum_distance_m=RANGE_M,
                                             observer_elevation_m=OBSERVER_M)
        fp64, _ = oracle.march_all_passes(segments, [pyramid(grid), regional_pyramid],
                                          tile_column=tile.tile_column, tile_row=tile.tile_row,
                                          observer_elevation_m=OBSERVER_M, pixels=pixels,
                                          azimuths=azimuths, precision="f64")
        reference = np.degrees(np.arctan(fp64))
        for traversal in errors:
            got = values[traversal][i][pixels, azimuths].astype(np.float64)
            finite = np.isfinite(reference) & np.isfinite(got)
            errors[traversal].append(np.abs(got[finite] - reference[finite]))
    summary = {}
    for traversal, parts in errors.items():
        e = np.concatenate(parts)
        summary[traversal] = {"p99.9": float(np.quantile(e, 0.999)), "max": float(e.max()),
                              "mean": float(e.mean()), "rays": int(e.size)}
    return summary


GENERATE_SIDE = 512


def generate_benchmark(primary, regional, rank):
    """End to end through the public tile generator: the central 512 x 512
    crop of the site DEM (16 tiles) with the regional DEM, 200 km rays,
    .cbin files written (staged, fsynced, renamed) to a RAM-backed directory.
    Per-tile reference traversal vs batches of 16 with the skip ladder; wall
    clock, including segment building, encoding, D2H and the file writes."""
    import shutil
    import tempfile

    from lunarscout_b200.contract import DemGrid
    from lunarscout_b200.horizon import generate_horizons_from_grids

    offset = (primary.width - GENERATE_SIDE) // 2
    transform = primary.geo_transform.copy()
    transform[0] += offset * transform[1]
    transform[3] += offset * transform[5]
    crop = DemGrid(np.ascontiguousarray(primary.elevation_m[offset:offset + GENERATE_SIDE,
                                                            offset:offset + GENERATE_SIDE]),
                   transform, primary.projection)
    tiles = (GENERATE_SIDE // TILE) ** 2
    base = Path("/dev/shm") if Path("/dev/shm").is_dir() else None
    result = {"tiles": tiles, "rays": tiles * RAYS_PER_TILE, "format": ".cbin",
              "output": "RAM-backed directory" if base else "temporary directory"}
    for name, options in (("per_tile", {}), ("batched_ladder",
                                             {"batch_tiles": 16, "traversal": "ladder"})):
        folder = Path(tempfile.mkdtemp(prefix=f"ls200_{rank}_", dir=base))
        try:
            started = time.perf_counter()
            generate_horizons_from_grids(folder, [crop, regional], compress=True,
                                         maximum_distance_m=RANGE_M, **options)
            seconds = time.perf_counter() - started
            written = sum(1 for _ in folder.rglob("horizon_*.cbin"))
        finally:
            shutil.rmtree(folder, ignore_errors=True)
        result[name] = {"seconds": seconds, "tiles_written": written,
                        "rays_per_s": tiles * RAYS_PER_TILE / seconds}
    result["speedup_batched_vs_per_tile"] = (result["per_tile"]["seconds"]
                                             / result["batched_ladder"]["seconds"])
    return result


ADJOINT_FD_CELLS = 200


def adjoint_benchmark(session, args, rank):
    """The differentiable-lighting configuration: a 256 x 256 study area (4
    tiles) in the middle of a 2048 x 2048 DEM at 10 m (fBm + craters), 1440
    azimuths, 20 km rays, loss = weighted (uniform [0, 1], seeded) mean smooth
    sun fraction over 29.53 days at 2 h steps (355 times).  Times the forward
    (march with argmax checkpoints, sun directions, loss) and the adjoint, and
    checks central finite differences at +-0.05 m on 200 cells."""
    import torch

    from lunarscout_b200.adjoint import SunLossProblem
    from lunarscout_b200.synthetic import SyntheticDemSpec, sun_vectors, synthetic_dem

    dem = synthetic_dem(SyntheticDemSpec(2048, 10.0, craters=300, crater_max_m=4000.0, seed=31))
    tiles = [(896, 896), (1024, 896), (896, 1024), (1024, 1024)]
    rng = np.random.default_rng(32 + rank)
    weights = rng.uniform(0.0, 1.0, size=(len(tiles), TILE, TILE)).astype(np.float32)
    vectors = sun_vectors(np.arange(355, dtype=np.float64) * 2.0)
    problem = SunLossProblem(session, [dem], tiles, weights, vectors,
                             maximum_distance_m=20_000.0, observer_elevation_m=OBSERVER_M,
                             azimuth_count=AZIMUTHS, traversal="ladder")
    heights = torch.from_numpy(dem.elevation_m).cuda()
    problem.forward_value([heights])
    problem.backward_value(1.0)
    forward, backward, walls = [], [], []
    for _ in range(3):
        started = time.perf_counter()
        loss = problem.forward_value()
        problem.backward_value(1.0)
        walls.append(time.perf_counter() - started)
        forward.append(problem.last_seconds["forward_march"]
                       + problem.last_seconds["forward_lighting"])
        backward.append(problem.last_seconds["backward"])
    forward_s, backward_s = statistics.median(forward), statistics.median(backward)
    result = {
        "metric": "DEM adjoint / forward time (smooth sun fraction, 20 km, 1440 az)",
        "loss": loss, "forward_ms": 1000.0 * forward_s, "backward_ms": 1000.0 * backward_s,
        "adjoint_over_forward": backward_s / forward_s,
        "forward_plus_adjoint_over_forward": (forward_s + backward_s) / forward_s,
        "wall_ms_forward_and_backward": 1000.0 * statistics.median(walls),
        "rays": len(tiles) * TILE * TILE * AZIMUTHS, "time_steps": len(vectors),
        "disk_radius_deg": problem.disk_radius_deg,
        "model": "smooth disk fraction (differentiable model, not the reference's 16-slice "
                 "fraction)",
    }
    if not args.skip_cpu:
        problem.forward_value([heights])
        problem.replay_value()
        (grad,) = problem.backward_value(1.0)
        grad = grad.cpu().numpy()
        magnitude = np.abs(grad).ravel()
        live = np.flatnonzero(magnitude > 1e-3 * magnitude.max())
        cells = rng.choice(live, min(ADJOINT_FD_CELLS, live.size), replace=False)
        observer = np.zeros(grad.shape, dtype=bool)
        observer[896:1152, 896:1152] = True
        errors = {"terrain": [], "observer": []}
        for index in cells:
            y, x = divmod(int(index), dem.width)
            h = heights.clone()
            h[y, x] += 0.05
            plus = problem.replay_value([h])
            h[y, x] -= 0.1
            minus = problem.replay_value([h])
            error = abs((plus - minus) / 0.1 - grad[y, x]) / abs(grad[y, x])
            errors["observer" if observer[y, x] else "terrain"].append(error)
        problem.set_heights([heights])
        summary = {}
        for kind, values in errors.items():
            if values:
                v = np.array(values)
                summary[kind] = {"cells": int(v.size), "median_rel": float(np.median(v)),
                                 "p90_rel": float(np.quantile(v, 0.9)),
                                 "within_1e-3": float(np.mean(v <= 1e-3))}
        result["finite_differences_0.05m_fixed_sampling"] = summary
    problem.close()
    return result


SENSITIVITY_SIDE = 8192
SENSITIVITY_BATCH = 4
SENSITIVITY_STEPS = 26281  # 3 years at 1 h


def sensitivity_benchmark(session, regional, args, rank):
    """A slice of the large batched sensitivity run: an 8192 x 8192 primary
    at 5 m (the site recipe, 2400 craters) with the regional DEM, 8 tiles
    around the centre, 200 km rays, 3 years of hourly Sun vectors.
    Horizons by the persistent ladder march, PSR over all 26,281 vectors,
    weights 1 within 500 m of each tile's PSR boundary, then the streamed
    adjoint of the weighted mean smooth sun fraction in batches of 4 tiles
    (the argmax checkpoints of one batch resident at a time)."""
    import ctypes

    import torch

    from lunarscout_b200 import _native, synthetic
    from lunarscout_b200.adjoint import StreamedSunLoss, psr_boundary_weights
    from lunarscout_b200.contract import projection_array
    from lunarscout_b200.cuda_backend import SiteTile
    from lunarscout_b200.lightmap_cuda import DeviceVectors

    started = time.perf_counter()
    primary = synthetic.site_dem(SENSITIVITY_SIDE, 5.0, craters=2400, seed=5)
    build_s = time.perf_counter() - started
    centre = SENSITIVITY_SIDE // 2
    tiles = [(centre + dx * TILE, centre + dy * TILE) for dy in (-1, 0) for dx in (-2, -1, 0, 1)]
    count = len(tiles)
    plane = TILE * TILE
    vectors = synthetic.sun_vectors(np.arange(SENSITIVITY_STEPS, dtype=np.float64))
    dems = [session.upload_dem_grid(primary), session.upload_dem_grid(regional)]
    horizons = torch.empty((count, plane, AZIMUTHS), dtype=torch.float32, device="cuda")
    site_tiles = [SiteTile(tuple(dems), tx, ty, RANGE_M, OBSERVER_M) for tx, ty in tiles]
    session.march_sites(site_tiles, device_out=horizons.data_ptr(), traversal="ladder",
                        degrees=True)
    _, march_s = session.march_sites(site_tiles, device_out=horizons.data_ptr(),
                                     traversal="ladder", degrees=True)
    patches = torch.stack([torch.from_numpy(np.ascontiguousarray(
        primary.elevation_m[ty:ty + TILE, tx:tx + TILE])) for tx, ty in tiles]).cuda()
    geo = np.ascontiguousarray(np.repeat(primary.geo_transform[None, :], count, 0))
    proj = np.ascontiguousarray(np.repeat(projection_array(primary.projection)[None, :],
                                          count, 0))
    windows = np.array([(tx, ty, TILE, TILE) for tx, ty in tiles], dtype=np.int32)
    table = DeviceVectors(session.context, vectors.astype(np.float32))
    frames = torch.empty(count * plane * 12, dtype=torch.float32, device="cuda")
    psr = torch.empty((count, plane), dtype=torch.uint8, device="cuda")
    lib = _native.library()

    def psr_launch():
        _native.check(lib.ls200_lighting_device(
            session.context, count, ctypes.c_void_p(patches.data_ptr()), geo.ctypes.data,
            proj.ctypes.data, windows.ctypes.data, ctypes.c_void_p(horizons.data_ptr()),
            table.handle, 0, SENSITIVITY_STEPS, 3, ctypes.c_void_p(frames.data_ptr()),
            ctypes.c_void_p(psr.data_ptr())))

    psr_launch()
    torch.cuda.synchronize()
    begin, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    begin.record()
    psr_launch()
    end.record()
    torch.cuda.synchronize()
    psr_s = begin.elapsed_time(end) / 1000.0
    table.close()
    masks = psr.cpu().numpy().reshape(count, TILE, TILE)
    weights = np.stack([psr_boundary_weights(m, 5.0, 500.0) for m in masks])
    del horizons
    for dem in dems:
        dem.close()
    streamed = StreamedSunLoss(session, [primary, regional], tiles, weights, vectors,
                               batch_tiles=SENSITIVITY_BATCH, maximum_distance_m=RANGE_M,
                               observer_elevation_m=OBSERVER_M, azimuth_count=AZIMUTHS,
                               traversal="ladder")
    heights = [torch.from_numpy(primary.elevation_m).cuda(),
               torch.from_numpy(regional.elevation_m).cuda()]
    try:
        loss, grads = streamed.value_and_gradient(heights)
        seconds = dict(streamed.last_seconds)
        free, total = torch.cuda.mem_get_info()
        nonzero = int(torch.count_nonzero(grads[0]))
    finally:
        streamed.close()
    forward_s = seconds["forward_march"] + seconds["forward_lighting"]
    rays = count * plane * AZIMUTHS
    return {
        "workload": "8 tiles of an 8192x8192 5 m primary + 240 m regional, 200 km rays, "
                    "3 years hourly (26,281 Sun vectors)",
        "tiles": count, "batch_tiles": SENSITIVITY_BATCH, "time_steps": SENSITIVITY_STEPS,
        "dem_build_s": build_s,
        "march_rays_per_s": rays / march_s,
        "psr_px_steps_per_s": count * plane * SENSITIVITY_STEPS / psr_s,
        "psr_fraction": float((masks > 0).mean()),
        "weighted_fraction": float(weights.mean()),
        "loss": loss, "forward_s": forward_s, "backward_s": seconds["backward"],
        "adjoint_over_forward": seconds["backward"] / forward_s,
        "gradient_nonzero_cells": nonzero,
        "device_memory_in_use_gb": (total - free) / 1e9,
        "memory_note": "cudaMemGetInfo after the run; the library keeps its largest buffers, "
                       "so this includes the run's peak",
    }


def run_ours(args):
    import torch
    import torch.distributed as dist

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    from lunarscout_b200.cuda_backend import CudaSession
    from lunarscout_b200._native import pinned_empty

    primary, regional = build_dems()
    session = CudaSession(local)
    # One explicit stream for torch and the library: the timing events are
    # recorded on the stream the kernels are launched on.
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    session.set_stream(stream.cuda_stream)
    dems = [session.upload_dem_grid(primary), session.upload_dem_grid(regional)]
    centers = (TILE // 8 + 2) ** 2
    total_steps = args.warmup + args.steps
    tiles = tile_schedule(rank, world, total_steps)
    segment_shape = (AZIMUTHS, centers, 2, 18)
    segments = []
    started = time.perf_counter()
    for tile_row, tile_column in tiles:
        buffer = torch.empty(segment_shape, dtype=torch.float32, device="cuda")
        session.generate_segments_device(dems, buffer.data_ptr(), tile_column=tile_column,
                                         tile_row=tile_row, azimuth_count=AZIMUTHS,
                                         maximum_distance_m=RANGE_M,
                                         observer_elevation_m=OBSERVER_M)
        segments.append(buffer)
    torch.cuda.synchronize()
    segment_seconds = (time.perf_counter() - started) / total_steps
    output = torch.empty((TILE * TILE, AZIMUTHS), dtype=torch.float32, device="cuda")

    def step(k, pass_seconds=None):
        tile_row, tile_column = tiles[k]
        session.march_all_passes_device(segments[k].data_ptr(), AZIMUTHS, centers, dems,
                                        tile_column=tile_column, tile_row=tile_row,
                                        observer_elevation_m=OBSERVER_M,
                                        device_out=output.data_ptr(), pass_seconds=pass_seconds)

    # Algorithmic work of the timed tiles: one counted (diagnostic) launch each.
    session.set_counting(True)
    visits = samples = ray_steps = 0
    for k in range(args.warmup, total_steps):
        step(k)
        torch.cuda.synchronize()
        v, s, n = session.last_counters()
        visits, samples, ray_steps = visits + v, samples + s, ray_steps + n
    session.set_counting(False)

    for k in range(args.warmup):
        step(k)
    torch.cuda.synchronize()

    sampler = ClockSampler(local)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    sampler.start()
    time.sleep(0.3)
    start_event = torch.cuda.Event(enable_timing=True)
    end_event = torch.cuda.Event(enable_timing=True)
    pass_times = []
    start_event.record(stream)
    for k in range(args.warmup, total_steps):
        seconds = np.zeros(2, dtype=np.float64)
        step(k, seconds)
        pass_times.append(seconds)
    end_event.record(stream)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    elapsed = max_over_ranks(start_event.elapsed_time(end_event) / 1000.0, world)
    if world > 1:
        dist.barrier()
    rays = world * args.steps * RAYS_PER_TILE
    value = rays / elapsed

    # End to end through the drop-in session call with pinned host buffers.
    e2e_value = None
    h2d = int(np.prod(segment_shape)) * 4
    d2h = TILE * TILE * AZIMUTHS * 4
    from lunarscout_b200.contract import PyramidArrays

    class _Pyr:  # the session's resident-pyramid cache keys on identity
        pass

    e2e_session = CudaSession(local)
    host_pyramids = []
    for dem in (primary, regional):
        p = e2e_session.build_max_pyramid(dem)
        host_pyramids.append(p)
    host_segments = [pinned_empty(segment_shape, np.float32) for _ in range(2)]
    for i in range(2):
        host_segments[i][...] = segments[args.warmup + i].cpu().numpy()
    e2e_session.subpatch_hierarchical_all_passes(host_segments[0], host_pyramids,
                                                 tile_column=tiles[args.warmup][1],
                                                 tile_row=tiles[args.warmup][0],
                                                 tile_width=TILE, tile_height=TILE,
                                                 subpatch_size=8)
    e2e_steps = max(2, min(args.steps, 6))
    if world > 1:
        dist.barrier()
    started = time.perf_counter()
    for k in range(e2e_steps):
        index = args.warmup + (k % 2)
        e2e_session.subpatch_hierarchical_all_passes(
            host_segments[k % 2], host_pyramids, tile_column=tiles[index][1],
            tile_row=tiles[index][0], tile_width=TILE, tile_height=TILE, subpatch_size=8)
    e2e_elapsed = max_over_ranks(time.perf_counter() - started, world)
    e2e_value = world * e2e_steps * RAYS_PER_TILE / e2e_elapsed
    e2e_session.close()

    lighting = lighting_benchmark(session, dems, segments, tiles, primary, args, world, rank)
    del segments
    multisite = None if args.skip_multisite else multisite_benchmark(session, stream, args,
                                                                     world, rank)
    adjoint = None if args.skip_adjoint else adjoint_benchmark(session, args, rank)
    sensitivity = (None if args.skip_sensitivity or world > 1
                   else sensitivity_benchmark(session, regional, args, rank))
    # The public generator runs on device 0 (as the reference's does): 1 GPU only.
    generate = (None if args.skip_generate or world > 1
                else generate_benchmark(primary, regional, rank))

    fp32_peak = session.fp32_probe()
    pass_times = np.array(pass_times)
    march_seconds = float(pass_times.sum()) / (2 * args.steps)  # per launch
    flops = (FLOPS_PER_STEP * ray_steps + FLOPS_PER_VISIT * visits
             + FLOPS_PER_SAMPLE * samples) / (2 * args.steps)
    achieved = flops / march_seconds / 1e12
    gathered = (BYTES_PER_VISIT * visits + BYTES_PER_SAMPLE * samples) / (2 * args.steps)

    cpu = None
    if rank == 0 and world == 1 and not args.skip_cpu:
        rate, threads, rays_cpu, secs = cpu_sample_rate(primary, regional, tiles[args.warmup:],
                                                        seconds_target=args.cpu_seconds)
        cpu = {"value": rate, "unit": "rays/s", "cores": threads, "kind": "port",
               "sample": f"{rays_cpu} random rays of the first timed tile, both DEM passes "
                         f"({secs:.1f} s)"}
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "rays/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1000.0 * elapsed / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic",
            "config": workload_config(),
            "roofline": {
                "bound": "fp32", "kernel": "march_pass_kernel",
                "achieved": achieved, "peak": fp32_peak, "unit": "TFLOP/s",
                "frac": achieved / fp32_peak,
                "peak_source": "FP32 FMA probe measured in this run (no FP32 entry in "
                               "MEASURED_PEAKS.json)",
                "traffic": profiled_traffic("march_pass_kernel_site_tile.md"),
                "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one "
                                  "pass-0 launch (profiles/march_pass_kernel_site_tile.md)",
                "algorithmic_flops_per_launch": flops,
                "gathered_bytes_per_launch": gathered,
                "launch_ms": march_seconds * 1000.0,
                "node_visits_per_ray": visits / (args.steps * RAYS_PER_TILE),
                "ray_steps_per_ray": ray_steps / (args.steps * RAYS_PER_TILE),
                "level0_samples_per_ray": samples / (args.steps * RAYS_PER_TILE),
            },
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": "rays/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "gpu_launches": 3 * args.steps,
            "clocks": clocks,
            "segment_generation_ms_per_tile": segment_seconds * 1000.0,
            "lightmap": lighting,
            "multisite": multisite,
            "adjoint": adjoint,
            "generate_horizons": generate,
            "sensitivity": sensitivity,
        }
        print(json.dumps(line), flush=True)
    session.close()
    if world > 1:
        dist.destroy_process_group()


def run_profile_case():
    """One site-scale tile marched twice (launches 3-4 are the second step's
    two passes); used under ncu, never timed."""
    import torch
    from lunarscout_b200.cuda_backend import CudaSession

    primary, regional = build_dems()
    session = CudaSession(0)
    dems = [session.upload_dem_grid(primary), session.upload_dem_grid(regional)]
    (tile_row, tile_column), = tile_schedule(0, 1, 1)
    centers = (TILE // 8 + 2) ** 2
    segments = torch.empty((AZIMUTHS, centers, 2, 18), dtype=torch.float32, device="cuda")
    output = torch.empty((TILE * TILE, AZIMUTHS), dtype=torch.float32, device="cuda")
    session.generate_segments_device(dems, segments.data_ptr(), tile_column=tile_column,
                                     tile_row=tile_row, azimuth_count=AZIMUTHS,
                                     maximum_distance_m=RANGE_M,
                                     observer_elevation_m=OBSERVER_M)
    for _ in range(2):
        session.march_all_passes_device(segments.data_ptr(), AZIMUTHS, centers, dems,
                                        tile_column=tile_column, tile_row=tile_row,
                                        observer_elevation_m=OBSERVER_M,
                                        device_out=output.data_ptr())
    session.synchronize()
    # Lighting on the same tile: one year of hourly sun-fraction bytes, twice.
    import ctypes

    from lunarscout_b200 import _native, synthetic
    from lunarscout_b200.contract import projection_array
    from lunarscout_b200.lightmap_cuda import DeviceVectors

    session.march_all_passes_device(segments.data_ptr(), AZIMUTHS, centers, dems,
                                    tile_column=tile_column, tile_row=tile_row,
                                    observer_elevation_m=OBSERVER_M,
                                    device_out=output.data_ptr(), degrees=True)
    patch = torch.from_numpy(np.ascontiguousarray(
        primary.elevation_m[tile_row:tile_row + TILE, tile_column:tile_column + TILE])).cuda()
    vectors = synthetic.sun_vectors(
        synthetic.hours_between("2030-01-01T00", "2031-01-01T00", 1.0)).astype(np.float32)
    table = DeviceVectors(session.context, vectors)
    frames = torch.empty(TILE * TILE * 12, dtype=torch.float32, device="cuda")
    out = torch.empty((len(vectors), TILE * TILE), dtype=torch.uint8, device="cuda")
    geo = np.ascontiguousarray(primary.geo_transform[None, :])
    proj = np.ascontiguousarray(projection_array(primary.projection)[None, :])
    window = np.array([[tile_column, tile_row, TILE, TILE]], dtype=np.int32)
    torch.cuda.synchronize()
    for _ in range(2):
        _native.check(_native.library().ls200_lighting_device(
            session.context, 1, ctypes.c_void_p(patch.data_ptr()), geo.ctypes.data,
            proj.ctypes.data, window.ctypes.data, ctypes.c_void_p(output.data_ptr()),
            table.handle, 0, len(vectors), 1, ctypes.c_void_p(frames.data_ptr()),
            ctypes.c_void_p(out.data_ptr())))
    session.synchronize()
    table.close()
    session.close()
    log("[bench] profile case done")


def run_profile_multisite():
    """Four tiles of the multi-site batch through the persistent march, exact
    traversal then skip ladder (launches 2 and 4 are the marches); used under
    ncu, never timed."""
    import torch

    from lunarscout_b200 import synthetic
    from lunarscout_b200.cuda_backend import CudaSession, SiteTile

    specs = synthetic.multisite_specs(SITES)[:4]
    grids = [synthetic.synthetic_dem(spec) for spec in specs]
    regional = synthetic.polar_regional_dem()
    session = CudaSession(0)
    regional_dev = session.upload_dem_grid(regional)
    tiles = []
    for grid in grids:
        dev = session.upload_dem_grid(grid)
        tiles.append(SiteTile((dev, regional_dev), (grid.width // 2 // TILE) * TILE,
                              (grid.height // 2 // TILE) * TILE, RANGE_M, OBSERVER_M))
    out = torch.empty(len(tiles) * RAYS_PER_TILE, dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    for traversal in ("exact", "ladder"):
        session.march_sites(tiles, device_out=out.data_ptr(), azimuth_count=AZIMUTHS,
                            traversal=traversal, degrees=True)
    session.close()
    log("[bench] multisite profile case done")


def main():
    parser = argparse.ArgumentParser()
    parser.add_argument("--gpus", type=int, default=1)
    parser.add_argument("--steps", type=int, default=10)
    parser.add_argument("--warmup", type=int, default=3)
    parser.add_argument("--impl", choices=("ours", "reference"), default="ours")
    parser.add_argument("--cpu-seconds", type=float, default=12.0)
    parser.add_argument("--reference-seconds", type=float, default=8.0)
    parser.add_argument("--skip-cpu", action="store_true")
    parser.add_argument("--skip-multisite", action="store_true",
                        help="leave out the uneven multi-site batched-vs-plain leg")
    parser.add_argument("--skip-adjoint", action="store_true",
                        help="leave out the DEM-adjoint (differentiable lighting) leg")
    parser.add_argument("--skip-generate", action="store_true",
                        help="leave out the end-to-end tile-generator leg")
    parser.add_argument("--skip-sensitivity", action="store_true",
                        help="leave out the 8192^2 streamed-adjoint sensitivity slice")
    parser.add_argument("--profile", nargs="?", const="site", choices=("site", "multisite"),
                        help="small profiling case, no timing: 'site' = one site-scale tile "
                             "(two march steps, two lighting launches); 'multisite' = four "
                             "tiles through the persistent march (exact, then ladder)")
    args = parser.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.profile == "multisite":
        run_profile_multisite()
    elif args.profile:
        run_profile_case()
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
