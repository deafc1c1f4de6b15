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


def profiled_value(name: str, key: str):
    """A `key: value` figure recorded by a committed ncu summary, if any."""
    path = ROOT / "profiles" / name
    try:
        for line in path.read_text().splitlines():
            if line.startswith(key + ":"):
                return float(line.split(":", 1)[1])
    except (OSError, ValueError):
        return None
    return None


def profiled_traffic(name: str):
    """DRAM bytes per launch recorded by the committed ncu summary, if any."""
    value = profiled_value(name, "dram_bytes_per_launch")
    return None if value is None else int(value)


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


class CpuMarchSample:
    """The oracle's C restatement of the march (all host threads) on random
    rays of one site-scale tile, both DEM passes: pyramids and segments are
    built once, then each call marches a fresh random ray sample."""

    def __init__(self, primary, regional, tile, threads=None):
        import oracle
        from oracle import segments as oseg
        from lunarscout_b200.contract import PyramidArrays, map_parameters, projection_parameters

        self.oracle = oracle
        self.pyramids = []
        for dem in (primary, regional):
            mips, levels = oracle.build_pyramid(dem.elevation_m)
            self.pyramids.append(PyramidArrays(dem.elevation_m, mips, levels,
                                               map_parameters(dem), projection_parameters(dem)))
        self.threads = threads or oracle.default_threads()
        self.tile_row, self.tile_column = tile
        self.segments = oseg.build_segments(
            [primary, regional], tile_column=self.tile_column, tile_row=self.tile_row,
            tile_width=TILE, azimuth_count=AZIMUTHS, maximum_distance_m=RANGE_M,
            observer_elevation_m=OBSERVER_M, threads=self.threads)
        self.rng = np.random.default_rng(7)

    def run(self, rays: int) -> float:
        """March `rays` random rays; returns the elapsed seconds."""
        pixels = self.rng.integers(0, TILE * TILE, size=rays).astype(np.int32)
        azimuths = self.rng.integers(0, AZIMUTHS, size=rays).astype(np.int32)
        started = time.perf_counter()
        self.oracle.march_all_passes(self.segments, self.pyramids, tile_column=self.tile_column,
                                     tile_row=self.tile_row, observer_elevation_m=OBSERVER_M,
                                     pixels=pixels, azimuths=azimuths, threads=self.threads)
        return time.perf_counter() - started


def cpu_sample_rate(primary, regional, tiles, seconds_target=12.0, threads=None):
    """Oracle march throughput (rays/s) on a bounded random ray sample."""
    sample = CpuMarchSample(primary, regional, tiles[0], threads)
    count, elapsed, rays = 256, 0.0, 0
    while elapsed < seconds_target:
        took = sample.run(count)
        elapsed += took
        rays += count
        if took < 1.0:
            count *= 4
    return rays / elapsed, sample.threads, rays, elapsed


# Rays of one reference-arm step: a bounded sample of the site-scale tile
# (about a second of CPU work on a 16-core host).
REFERENCE_STEP_RAYS = 1 << 17


def run_reference(args):
    """The reference algorithm on the host cores: each step marches a fresh
    random sample of REFERENCE_STEP_RAYS rays of the site-scale tile (both DEM
    passes) with the oracle's C restatement; value = rays / measured seconds
    per step, ms_per_step = the measured step time (median)."""
    rank, world, _ = dist_env()
    if rank != 0:
        return
    primary, regional = build_dems()
    sample = CpuMarchSample(primary, regional, tile_schedule(0, 1, 1)[0])
    per_step = []
    for step in range(args.warmup + args.steps):
        took = sample.run(REFERENCE_STEP_RAYS)
        if step >= args.warmup:
            per_step.append(took)
    step_seconds = statistics.median(per_step)
    value = REFERENCE_STEP_RAYS / step_seconds
    line = {
        "impl": "reference",
        "metric": METRIC, "value": value, "unit": "rays/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000.0 * step_seconds,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": workload_config(),
        "cpu_baseline": {"value": value, "unit": "rays/s", "cores": sample.threads,
                         "kind": "port",
                         "sample": f"each step: {REFERENCE_STEP_RAYS} random rays of a "
                                   f"site-scale tile, both DEM passes (a step of the GPU arm "
                                   f"is the whole tile, {RAYS_PER_TILE} rays)"},
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
        host_horizons = horizons[0].cpu().numpy().reshape(TILE, TILE, AZIMUTHS)
        tile_row, tile_column = tiles[picks[0]]
        reference = reference_cpu_lighting(primary, host_horizons, tile_row, tile_column,
                                           synthetic.sun_vectors(hours))
        if reference is not None:
            result["cpu_baseline"] = reference["lightmap"]
            result["reference_cpu_psr"] = reference["psr"]
        else:
            from oracle import products

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


def reference_cpu_lighting(primary, host_horizons, tile_row, tile_column, sun_vectors):
    """The reference's own CPU lighting on the box's host cores:
    LightmapCpuSession (lightmap_cpu.py:193, Numba parallel) sun-fraction
    bytes of one tile over the year, and compute_psr_patch_reference
    (psr.py:94, NumPy per pixel) on a 32 x 32 window against the reduced
    vectors.  None when the reference is not installed."""
    runtime = reference_runtime()
    if runtime is None:
        return None
    import numba

    runtime.import_reference()
    from lunarscout._numba_horizon.lightmap_cpu import LightmapCpuSession
    from lunarscout._numba_horizon.psr import (compute_psr_patch_reference,
                                               reduce_sun_vectors_for_psr)

    dem = reference_dem(primary)
    horizons = np.where(np.isneginf(host_horizons), np.float32(-50.0), host_horizons)
    session = LightmapCpuSession(time_batch_size=32)
    tile = dict(tile_y=tile_row, tile_x=tile_column)
    for _ in session.iter_patch_tiles(dem, horizons, sun_vectors[:64], **tile):
        pass  # compiles the Numba kernels
    started = time.perf_counter()
    for _ in session.iter_patch_tiles(dem, horizons, sun_vectors, **tile):
        pass
    lightmap_s = time.perf_counter() - started
    reduced, _ = reduce_sun_vectors_for_psr(dem, sun_vectors)
    window = 32
    started = time.perf_counter()
    compute_psr_patch_reference(dem, horizons, reduced, valid_height=window,
                                valid_width=window, **tile)
    psr_s = time.perf_counter() - started
    return {
        "lightmap": {"value": TILE * TILE * len(sun_vectors) / lightmap_s, "unit": "px·steps/s",
                     "cores": numba.config.NUMBA_NUM_THREADS, "kind": "reference",
                     "sample": f"LightmapCpuSession.iter_patch_tiles, one tile x "
                               f"{len(sun_vectors)} hourly steps ({lightmap_s:.1f} s)"},
        "psr": {"value": window * window * len(reduced) / psr_s,
                "unit": "px·reduced vectors/s", "cores": 1, "kind": "reference",
                "sample": f"compute_psr_patch_reference, {window}x{window} px x "
                          f"{len(reduced)} reduced vectors ({psr_s:.1f} s)"},
    }


SITES = 64
WARMUP_TILES = 16  # the warm-up batch: one tile of each of the first 16 sites
TUNE_TILES = 4
MULTISITE_PARITY_RAYS = 20_000


def distance_over_every_ray(a, b, bin_deg=1e-5, bins=100_000):
    """p99.9 (to the histogram's bin width) and max of |a - b| (degrees) over
    every finite ray of two degree batches [tiles, pixels, azimuths], with
    the (tile, pixel, azimuth) of the max, the rays beyond 0.01 and 1 deg,
    and whether the -inf rays agree."""
    import torch

    counts = torch.zeros(bins + 1, dtype=torch.int64, device=a.device)
    largest, at, same_inf, total, over = 0.0, None, True, 0, [0, 0]
    for t in range(a.shape[0]):
        finite = torch.isfinite(a[t]) & torch.isfinite(b[t])
        same_inf &= bool(torch.equal(torch.isfinite(a[t]), torch.isfinite(b[t])))
        full = torch.where(finite, (a[t].double() - b[t].double()).abs(),
                           torch.zeros((), dtype=torch.float64, device=a.device))
        d = full[finite]
        if d.numel() == 0:
            continue
        total += d.numel()
        over[0] += int((d > 0.01).sum())
        over[1] += int((d > 1.0).sum())
        worst = int(torch.argmax(full))
        if float(full.view(-1)[worst]) > largest:
            largest = float(full.view(-1)[worst])
            at = (t, worst // full.shape[1], worst % full.shape[1])
        counts += torch.bincount((d / bin_deg).long().clamp(max=bins), minlength=bins + 1)
    cumulative = torch.cumsum(counts, 0)
    rank = int(math.ceil(0.999 * int(cumulative[-1])))
    index = int(torch.searchsorted(cumulative, torch.tensor([rank], device=a.device)))
    return {"p99.9": (index + 1) * bin_deg, "max": largest, "max_at": at, "rays": total,
            "over_0.01": over[0], "over_1": over[1], "inf_rays_agree": same_inf}


def multisite_benchmark(session, stream, args, world, rank):
    """The uneven multi-site workload (64 sites, sides 256-2048 px at 5-40 m,
    latitudes -83 to -89.5, one polar 240 m regional DEM, 200 km rays): the
    timed batch is one tile of EVERY site (64 tiles) in one launch.  Plain =
    per-tile device segments + per-pass launches + transpose; batched = one
    persistent work-stealing launch over the whole batch (reference
    traversal, skip ladder, and the ladder in the relative FP32 arithmetic),
    launch configuration chosen by the autotuner.  Degrees in HBM, CUDA
    events; a smaller warm-up batch precedes each timed one."""
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

    def random_tile(site):
        grid = grids[site]
        tx = int(rng.integers(0, (grid.width + TILE - 1) // TILE)) * TILE
        ty = int(rng.integers(0, (grid.height + TILE - 1) // TILE)) * TILE
        return SiteTile((site_devs[site], regional_dev), tx, ty, RANGE_M, OBSERVER_M)

    warmup = [random_tile(site) for site in range(WARMUP_TILES)]
    batch = [random_tile(site) for site in range(SITES)]

    def valid(tile, site):
        grid = grids[site]
        return (min(TILE, grid.width - tile.tile_column),
                min(TILE, grid.height - tile.tile_row))

    timed_rays = sum(w * h for w, h in (valid(t, s) for s, t in enumerate(batch))) * AZIMUTHS
    centers = (TILE // 8 + 2) ** 2
    segments = torch.empty(AZIMUTHS * centers * 2 * 18, dtype=torch.float32, device="cuda")
    outputs = {name: torch.empty((SITES, TILE * TILE, AZIMUTHS), dtype=torch.float32,
                                 device="cuda")
               for name in ("exact", "ladder", "relative-ladder")}
    torch.cuda.synchronize()

    def plain(tiles, out):
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

    splits = {}  # traversal -> (segment + setup seconds, march seconds) of the timed call

    def batched(traversal):
        def run(tiles, out):
            splits[traversal] = session.march_sites(
                tiles, device_out=out.data_ptr(), azimuth_count=AZIMUTHS, traversal=traversal,
                degrees=True)
        return run

    def timed(run, out):
        run(warmup, out)
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record(stream)
        run(batch, out)
        end.record(stream)
        torch.cuda.synchronize()
        elapsed = max_over_ranks(start.elapsed_time(end) / 1000.0, world)
        return world * timed_rays / elapsed, elapsed

    # Each batched traversal runs with the launch configuration the autotuner
    # picks for it (the relative arithmetic holds more registers).
    tuned = {traversal: tune_batch(session, warmup[:TUNE_TILES],
                                   device_out=outputs[traversal].data_ptr(),
                                   azimuth_count=AZIMUTHS, traversal=traversal)
             for traversal in ("exact", "ladder", "relative-ladder")}
    values, seconds = {}, {}
    values["plain"], seconds["plain"] = timed(plain, outputs["exact"])
    for traversal in ("exact", "ladder", "relative-ladder"):
        session.set_batch_config(tuned[traversal].best)
        values[traversal], seconds[traversal] = timed(batched(traversal), outputs[traversal])
    result = {
        "metric": "multi-site horizon rays/s (uneven batch, 2 DEM passes, 200 km)",
        "unit": "rays/s",
        "plain_per_tile": values["plain"],
        "batched_exact": values["exact"],
        "batched_ladder": values["ladder"],
        "batched_relative_ladder": values["relative-ladder"],
        "speedup_batched_vs_plain": values["ladder"] / values["plain"],
        "speedup_relative_ladder_vs_plain": values["relative-ladder"] / values["plain"],
        "speedup_exact_vs_plain": values["exact"] / values["plain"],
        "seconds": seconds,
        "batched_split_seconds": {
            traversal: {"segments_and_setup": split[0], "march": split[1]}
            for traversal, split in splits.items()},
        "launch_config": {
            traversal: {"lanes_per_azimuth": result.best.lanes_per_azimuth,
                        "min_blocks": result.best.min_blocks,
                        "candidates_ms": {
                            f"lanes{c.lanes_per_azimuth}/blocks{c.min_blocks}": 1000.0 * t
                            for c, t in result.seconds.items()}}
            for traversal, result in tuned.items()},
        "launch_config_tuned_on": f"{TUNE_TILES} tiles of the warm-up batch",
        "sites": SITES, "tiles_per_launch": SITES, "warmup_tiles": WARMUP_TILES,
        "rays_timed_per_rank": timed_rays,
        "rays": "rays of pixels inside each site DEM (partial edge tiles count their valid part)",
        "every_ray_vs_exact_deg": {
            "ladder": distance_over_every_ray(outputs["ladder"], outputs["exact"]),
            "relative_ladder": distance_over_every_ray(outputs["relative-ladder"],
                                                       outputs["exact"]),
        },
    }
    if rank == 0 and world == 1 and not args.skip_cpu:
        result["parity"] = multisite_parity(session, grids, regional, batch, outputs)
        result["largest_distances_vs_fp64"] = {
            name: ray_against_fp64(session, grids, regional, batch, outputs,
                                   result["every_ray_vs_exact_deg"][name]["max_at"])
            for name in ("ladder", "relative_ladder")}
    del outputs["exact"], outputs["ladder"]
    result["pipeline"] = multisite_products(session, stream, grids, batch,
                                            outputs["relative-ladder"], args)
    for dem in site_devs + [regional_dev]:
        dem.close()
    return result


def ray_against_fp64(session, grids, regional, batch, outputs, at):
    """Each traversal's degrees and the FP64 restatement's at one ray
    (tile, pixel, azimuth) of the 64-site batch."""
    import oracle
    from lunarscout_b200.contract import PyramidArrays, map_parameters, projection_parameters

    if at is None:
        return None
    t, pixel, azimuth = (int(v) for v in at)
    tile, grid = batch[t], grids[t]
    pyramids = []
    for dem in (grid, regional):
        mips, levels = oracle.build_pyramid(dem.elevation_m)
        pyramids.append(PyramidArrays(dem.elevation_m, mips, levels, map_parameters(dem),
                                      projection_parameters(dem)))
    segments = session.generate_segments(list(tile.dems), tile_column=tile.tile_column,
                                         tile_row=tile.tile_row, azimuth_count=AZIMUTHS,
                                         maximum_distance_m=RANGE_M,
                                         observer_elevation_m=OBSERVER_M)
    fp64, _ = oracle.march_all_passes(segments, pyramids, tile_column=tile.tile_column,
                                      tile_row=tile.tile_row, observer_elevation_m=OBSERVER_M,
                                      pixels=np.array([pixel], np.int32),
                                      azimuths=np.array([azimuth], np.int32), precision="f64")
    values = {name: float(out[t, pixel, azimuth]) for name, out in outputs.items()}
    values["fp64"] = float(np.degrees(np.arctan(fp64[0])))
    values["ray"] = {"site": t, "pixel": pixel, "azimuth": azimuth}
    return values


def multisite_parity(session, grids, regional, batch, outputs):
    """The 64-site batch against the oracle on MULTISITE_PARITY_RAYS random
    rays spread over all tiles: the reference traversal against the FP32
    oracle and the relative ladder against its FP32 restatement, bit for
    bit; every traversal's distance from the FP64 restatement."""
    import torch

    import oracle
    from lunarscout_b200.contract import PyramidArrays, map_parameters, projection_parameters

    def pyramid(dem):
        mips, levels = oracle.build_pyramid(dem.elevation_m)
        return PyramidArrays(dem.elevation_m, mips, levels, map_parameters(dem),
                             projection_parameters(dem))

    regional_pyramid = pyramid(regional)
    rng = np.random.default_rng(9)
    per_tile = MULTISITE_PARITY_RAYS // len(batch) + 1
    bits = {"exact": True, "relative-ladder": True}
    errors = {name: [] for name in outputs}
    rays = 0
    for t, (tile, grid) in enumerate(zip(batch, grids)):
        width = min(TILE, grid.width - tile.tile_column)
        height = min(TILE, grid.height - tile.tile_row)
        pixels = (rng.integers(0, height, per_tile) * TILE
                  + rng.integers(0, width, per_tile)).astype(np.int32)
        azimuths = rng.integers(0, AZIMUTHS, per_tile).astype(np.int32)
        segments = session.generate_segments(list(tile.dems), tile_column=tile.tile_column,
                                             tile_row=tile.tile_row, azimuth_count=AZIMUTHS,
                                             maximum_distance_m=RANGE_M,
                                             observer_elevation_m=OBSERVER_M)
        pyramids = [pyramid(grid), regional_pyramid]
        common = dict(tile_column=tile.tile_column, tile_row=tile.tile_row,
                      observer_elevation_m=OBSERVER_M, pixels=pixels, azimuths=azimuths)
        index = (torch.from_numpy(pixels.astype(np.int64)).cuda(),
                 torch.from_numpy(azimuths.astype(np.int64)).cuda())
        got = {name: out[t][index].cpu().numpy() for name, out in outputs.items()}
        expected = {
            "exact": oracle.march_all_passes(segments, pyramids, **common)[0],
            "relative-ladder": oracle.march_all_passes(
                segments, pyramids, mask=oracle.ladder_mask(0, 1) | oracle.OPT_RELATIVE,
                **common)[0],
        }
        for name, slopes in expected.items():
            # The batch writes degrees with the device's slope -> degree
            # conversion; apply the same conversion to the oracle's slopes.
            degrees = session.slopes_to_degrees(slopes.reshape(1, -1)).reshape(-1)
            bits[name] &= bool(np.array_equal(got[name], degrees))
        fp64 = np.degrees(np.arctan(oracle.march_all_passes(segments, pyramids,
                                                            precision="f64", **common)[0]))
        finite = np.isfinite(fp64)
        for name in outputs:
            errors[name].append(np.abs(got[name][finite].astype(np.float64) - fp64[finite]))
        rays += per_tile
    summary = {"rays": rays, "tiles": len(batch),
               "c3_bits_equal": bits["exact"],
               "c3_relative_ladder_bits_equal": bits["relative-ladder"],
               "error_vs_fp64_deg": {}}
    for name, parts in errors.items():
        e = np.concatenate(parts)
        summary["error_vs_fp64_deg"][name] = {
            "p99.9": float(np.quantile(e, 0.999)), "max": float(e.max()),
            "over_0.01": int((e > 0.01).sum())}
    return summary


def multisite_products(session, stream, grids, batch, horizons, args):
    """The multi-site products over two years of hourly steps (17,521) on the
    64 tiles of the multi-site batch, from the relative-ladder horizons left in
    HBM by the batched march: sun-fraction bytes, PSR against each site's reduced Sun
    vectors (the reduction over that site's DEM, on the device), and the
    Earth-visibility fraction.  The lightmap and PSR launches run eagerly and
    then as one replayed CUDA graph (one node per launch over the whole
    period); Earth visibility runs eagerly."""
    import ctypes

    import torch

    from lunarscout_b200 import _native, synthetic
    from lunarscout_b200.contract import projection_array
    from lunarscout_b200.graphs import DeviceGraph
    from lunarscout_b200.lightmap_cuda import DeviceVectors
    from lunarscout_b200.psr_cuda import reduce_vectors_on

    count = len(batch)
    plane = TILE * TILE
    hours = synthetic.hours_between("2030-01-01T00", "2032-01-01T00", 1.0)
    steps = len(hours)
    sun64, earth64 = synthetic.sun_vectors(hours), synthetic.earth_vectors(hours)
    sun = DeviceVectors(session.context, sun64.astype(np.float32))
    earth = DeviceVectors(session.context, earth64.astype(np.float32))
    patches = torch.zeros((count, TILE, TILE), dtype=torch.float32, device="cuda")
    geo = np.zeros((count, 6), dtype=np.float64)
    proj = np.zeros((count, 6), dtype=np.float64)
    windows = np.zeros((count, 4), dtype=np.int32)
    started = time.perf_counter()
    reduced = []
    for i, tile in enumerate(batch[:count]):
        grid = grids[i]
        vw = min(TILE, grid.width - tile.tile_column)
        vh = min(TILE, grid.height - tile.tile_row)
        patches[i, :vh, :vw] = torch.from_numpy(np.ascontiguousarray(
            grid.elevation_m[tile.tile_row:tile.tile_row + vh,
                             tile.tile_column:tile.tile_column + vw])).cuda()
        geo[i] = grid.geo_transform
        proj[i] = projection_array(grid.projection)
        windows[i] = (tile.tile_column, tile.tile_row, vw, vh)
        vectors, _ = reduce_vectors_on(session.context, grid, sun64)
        reduced.append(DeviceVectors(session.context, vectors.astype(np.float32)))
    reduction_seconds = time.perf_counter() - started
    # A ray with no terrain sample (-inf) is read as -50 deg, the value a
    # stored tile decodes to there.
    lit = horizons[:count]
    lit.masked_fill_(torch.isneginf(lit), -50.0)
    per_launch = 32
    frames = torch.empty(min(count, per_launch) * plane * 12, dtype=torch.float32,
                         device="cuda")
    light = torch.empty((count, steps, plane), dtype=torch.uint8, device="cuda")
    psr = torch.empty((count, plane), dtype=torch.uint8, device="cuda")
    visible = torch.empty((count, plane), dtype=torch.float32, device="cuda")
    lib = _native.library()
    groups = [(first, min(per_launch, count - first)) for first in range(0, count, per_launch)]

    def lighting(first, n, table, start, length, signal, target):
        _native.check(lib.ls200_lighting_device(
            session.context, n, ctypes.c_void_p(patches[first].data_ptr()),
            geo[first:].ctypes.data, proj[first:].ctypes.data, windows[first:].ctypes.data,
            ctypes.c_void_p(lit[first].data_ptr()), table.handle, start, length, signal,
            ctypes.c_void_p(frames.data_ptr()), ctypes.c_void_p(target)))

    def lightmap():
        for first, n in groups:
            lighting(first, n, sun, 0, steps, 1, light[first].data_ptr())

    def psr_all():
        for i in range(count):
            lighting(i, 1, reduced[i], 0, reduced[i].count, 3, psr[i].data_ptr())

    def visibility():
        for first, n in groups:
            _native.check(lib.ls200_earth_visibility_device(
                session.context, n, ctypes.c_void_p(patches[first].data_ptr()),
                geo[first:].ctypes.data, proj[first:].ctypes.data, windows[first:].ctypes.data,
                ctypes.c_void_p(lit[first].data_ptr()), earth.handle, ctypes.c_float(0.0),
                ctypes.c_void_p(visible[first].data_ptr())))

    events = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    torch.cuda.synchronize()
    events[0].record(stream)
    lightmap()
    events[1].record(stream)
    psr_all()
    events[2].record(stream)
    visibility()
    events[3].record(stream)
    torch.cuda.synchronize()
    lightmap_s = events[0].elapsed_time(events[1]) / 1000.0
    psr_s = events[1].elapsed_time(events[2]) / 1000.0
    visibility_s = events[2].elapsed_time(events[3]) / 1000.0
    graph = DeviceGraph.capture(session.context, lambda: (lightmap(), psr_all()))
    try:
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record(stream)
        graph.launch()
        end.record(stream)
        torch.cuda.synchronize()
        graph_s = start.elapsed_time(end) / 1000.0
        nodes = graph.nodes
    finally:
        graph.close()
    pixels = int(sum(int(w[2]) * int(w[3]) for w in windows))
    reduced_counts = [t.count for t in reduced]
    psr_px_steps = sum(int(w[2]) * int(w[3]) * c for w, c in zip(windows, reduced_counts))
    defined = torch.isfinite(visible)
    result = {
        "tiles": count, "of_batch_tiles": len(batch), "time_steps": steps,
        "lightmap_px_steps_per_s": pixels * steps / lightmap_s,
        "lightmap_seconds": lightmap_s,
        "psr_reduced_vectors_mean": float(np.mean(reduced_counts)),
        "psr_px_reduced_vectors_per_s": psr_px_steps / psr_s, "psr_seconds": psr_s,
        "psr_fraction": float((psr == 255).float().mean()),
        "vector_reduction_seconds_per_site": reduction_seconds / count,
        "earth_visibility_px_steps_per_s": pixels * steps / visibility_s,
        "earth_visibility_seconds": visibility_s,
        "earth_visibility_mean": float(visible[defined].mean()),
        "graph": {"nodes": nodes, "replay_seconds": graph_s,
                  "eager_seconds": lightmap_s + psr_s,
                  "replay_over_eager_throughput": (lightmap_s + psr_s) / graph_s,
                  "work": "lightmap (whole period per launch) + PSR per tile"},
        "work": "two years hourly: sun-fraction bytes, PSR over each site's reduced Sun "
                "vectors, Earth-visibility fraction (margin >= 0)",
    }
    for table in reduced + [sun, earth]:
        table.close()
    return result


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
    checks central finite differences (adjoint_finite_differences)."""
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
        result["finite_differences_fixed_sampling"] = adjoint_finite_differences(
            problem, heights, dem, rng)
    problem.close()
    return result


# Steps of the finite-difference check (m): the configured +-0.05 m, and two
# powers of two a factor 4 apart for the Richardson extrapolation.
FD_STEPS = (0.05, 2.0 ** -10, 2.0 ** -12)
FD_STRONGEST = 50


def adjoint_finite_differences(problem, heights, dem, rng):
    """Central differences of the replayed loss (the march's sampling held
    fixed) against the adjoint on ADJOINT_FD_CELLS random cells with a
    gradient and the FD_STRONGEST largest-gradient cells, split into the
    observers' own cells and terrain: at +-0.05 m, at 2^-12 m, and the
    Richardson extrapolation (16 D(2^-12) - D(2^-10)) / 15.  Each difference
    divides by the float32 heights' actual separation."""
    problem.forward_value([heights])
    problem.replay_value()
    (grad,) = problem.backward_value(1.0)
    grad = grad.cpu().numpy()
    magnitude = np.abs(grad).ravel()
    live = np.flatnonzero(magnitude > 1e-3 * magnitude.max())
    picks = {"random": rng.choice(live, min(ADJOINT_FD_CELLS, live.size), replace=False),
             "strongest": np.argsort(magnitude)[-FD_STRONGEST:]}
    observer = np.zeros(grad.shape, dtype=bool)
    observer[896:1152, 896:1152] = True

    def difference(y, x, step):
        h = heights.clone()
        base = float(heights[y, x])
        h[y, x] = base + step
        upper = float(h[y, x])
        plus = problem.replay_value([h])
        h[y, x] = base - step
        lower = float(h[y, x])
        minus = problem.replay_value([h])
        return (plus - minus) / (upper - lower)

    summary = {}
    for pick, cells in picks.items():
        errors = {"terrain": [], "observer": []}
        for index in cells:
            y, x = divmod(int(index), dem.width)
            d = [difference(y, x, step) for step in FD_STEPS]
            richardson = (16.0 * d[2] - d[1]) / 15.0
            g = grad[y, x]
            errors["observer" if observer[y, x] else "terrain"].append(
                [abs(d[0] - g) / abs(g), abs(d[2] - g) / abs(g), abs(richardson - g) / abs(g)])
        for kind, values in errors.items():
            if not values:
                continue
            v = np.array(values)
            summary[f"{pick}_{kind}"] = {
                "cells": int(len(v)),
                "median_rel_0.05m": float(np.median(v[:, 0])),
                "median_rel_2^-12m": float(np.median(v[:, 1])),
                "median_rel_richardson": float(np.median(v[:, 2])),
                "within_1e-3_richardson": float(np.mean(v[:, 2] <= 1e-3)),
                "p90_rel_richardson": float(np.quantile(v[:, 2], 0.9))}
    problem.set_heights([heights])
    return summary


SENSITIVITY_SIDE = 8192
SENSITIVITY_BATCH = 4
SENSITIVITY_STEPS = 26281  # 3 years at 1 h


def sensitivity_benchmark(session, regional, args, rank):
    """A slice of the large batched sensitivity run: an 8192 x 8192 primary
    at 5 m (the site recipe, 2400 craters) with the regional DEM, 8 tiles
    around the centre, 200 km rays, 3 years of hourly Sun and Earth vectors.
    Horizons by the persistent ladder march; PSR over the Sun vectors reduced
    over the DEM (as the PSR product does) and over all of them; the Sun+Earth
    mission-duration product (weekly candidate windows); weights 1 within
    500 m of each tile's PSR boundary, then the streamed adjoint of the
    weighted mean smooth sun fraction in batches of 4 tiles (the argmax
    checkpoints of one batch resident at a time).  Peak device memory is the
    high-water mark of the library's own allocations plus torch's."""
    import ctypes

    import torch

    from lunarscout_b200 import _native, synthetic
    from lunarscout_b200.adjoint import StreamedSunLoss, psr_boundary_weights
    from lunarscout_b200.contract import projection_array
    from lunarscout_b200.cuda_backend import SiteTile
    from lunarscout_b200.lightmap_cuda import DeviceVectors
    from lunarscout_b200.psr_cuda import reduce_vectors_on

    torch.cuda.synchronize()
    _native.memory_stats(session.device_id, reset_peak=True)
    torch.cuda.reset_peak_memory_stats()
    started = time.perf_counter()
    primary = synthetic.site_dem(SENSITIVITY_SIDE, 5.0, craters=2400, seed=5)
    build_s = time.perf_counter() - started
    centre = SENSITIVITY_SIDE // 2
    tiles = [(centre + dx * TILE, centre + dy * TILE) for dy in (-1, 0) for dx in (-2, -1, 0, 1)]
    count = len(tiles)
    plane = TILE * TILE
    hours = np.arange(SENSITIVITY_STEPS, dtype=np.float64)
    vectors = synthetic.sun_vectors(hours)
    earth_vectors = synthetic.earth_vectors(hours)
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
    started = time.perf_counter()
    reduced_vectors, reduced_indices = reduce_vectors_on(session.context, primary, vectors)
    reduction_s = time.perf_counter() - started
    table = DeviceVectors(session.context, vectors.astype(np.float32))
    reduced_table = DeviceVectors(session.context, reduced_vectors.astype(np.float32))
    earth = DeviceVectors(session.context, earth_vectors.astype(np.float32))
    frames = torch.empty(count * plane * 12, dtype=torch.float32, device="cuda")
    psr = torch.empty((count, plane), dtype=torch.uint8, device="cuda")
    psr_all = torch.empty((count, plane), dtype=torch.uint8, device="cuda")
    lib = _native.library()

    def psr_launch(vector_table, target):
        _native.check(lib.ls200_lighting_device(
            session.context, count, ctypes.c_void_p(patches.data_ptr()), geo.ctypes.data,
            proj.ctypes.data, windows.ctypes.data, ctypes.c_void_p(horizons.data_ptr()),
            vector_table.handle, 0, vector_table.count, 3, ctypes.c_void_p(frames.data_ptr()),
            ctypes.c_void_p(target.data_ptr())))

    def timed(run):
        run()
        torch.cuda.synchronize()
        begin, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        begin.record()
        run()
        end.record()
        torch.cuda.synchronize()
        return begin.elapsed_time(end) / 1000.0

    psr_s = timed(lambda: psr_launch(reduced_table, psr))
    psr_all_s = timed(lambda: psr_launch(table, psr_all))
    # Sun + Earth mission duration: condition = fraction >= 0.5 and Earth
    # margin >= 0, 30-day candidate start windows (36 over the three years;
    # the device reducer takes up to 64), 1 h samples.
    window = 30 * 24
    starts = np.arange(0, SENSITIVITY_STEPS - window, window, dtype=np.int32)
    start_windows = np.ascontiguousarray(np.stack([starts, starts + window], axis=1))
    sample_hours = np.ones(SENSITIVITY_STEPS, dtype=np.float64)
    mission = torch.empty((count, len(starts), plane), dtype=torch.float32, device="cuda")

    def mission_launch():
        _native.check(lib.ls200_mission_duration_device(
            session.context, count, ctypes.c_void_p(patches.data_ptr()), geo.ctypes.data,
            proj.ctypes.data, windows.ctypes.data, ctypes.c_void_p(horizons.data_ptr()),
            table.handle, earth.handle, ctypes.c_float(0.5), ctypes.c_float(0.0),
            sample_hours.ctypes.data, start_windows.ctypes.data, len(starts), 0,
            ctypes.c_void_p(mission.data_ptr())))

    mission_s = timed(mission_launch)
    for t in (table, reduced_table, earth):
        t.close()
    masks = psr.cpu().numpy().reshape(count, TILE, TILE)
    band = None
    if rank == 0 and not args.skip_cpu:
        band = psr_band(primary, horizons[0], reduced_vectors, masks[0], tiles[0])
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
        nonzero = int(torch.count_nonzero(grads[0]))
    finally:
        streamed.close()
    torch.cuda.synchronize()
    _, library_peak = _native.memory_stats(session.device_id)
    torch_peak = torch.cuda.max_memory_allocated()
    forward_s = seconds["forward_march"] + seconds["forward_lighting"]
    rays = count * plane * AZIMUTHS
    return {
        "workload": "8 tiles of an 8192x8192 5 m primary + 240 m regional, 200 km rays, "
                    f"3 years hourly ({SENSITIVITY_STEPS:,} Sun and Earth vectors)",
        "tiles": count, "batch_tiles": SENSITIVITY_BATCH, "time_steps": SENSITIVITY_STEPS,
        "dem_build_s": build_s,
        "march_rays_per_s": rays / march_s,
        "psr_reduced_vectors": int(len(reduced_indices)),
        "psr_vector_reduction_s": reduction_s,
        "psr_px_reduced_vectors_per_s": count * plane * len(reduced_indices) / psr_s,
        "psr_ms_per_tile": 1000.0 * psr_s / count,
        "psr_all_vectors_px_steps_per_s": count * plane * SENSITIVITY_STEPS / psr_all_s,
        "psr_fraction": float((masks > 0).mean()),
        "psr_fraction_all_vectors": float((psr_all.cpu().numpy() > 0).mean()),
        "psr_band": band,
        "mission_sun_earth": {"windows": int(len(starts)), "window_hours": window,
                              "px_steps_per_s": count * plane * SENSITIVITY_STEPS / mission_s,
                              "seconds": mission_s,
                              "mean_longest_hours": float(mission.mean())},
        "weighted_fraction": float(weights.mean()),
        "loss": loss, "forward_s": forward_s, "backward_s": seconds["backward"],
        "adjoint_over_forward": seconds["backward"] / forward_s,
        "gradient_nonzero_cells": nonzero,
        "peak_device_memory_gb": {
            "library_high_water": library_peak / 1e9,
            "torch_high_water": torch_peak / 1e9,
            "bound": (library_peak + torch_peak) / 1e9,
            "note": "high-water marks of the library's own allocations "
                    "(ls200_memory_stats) and of torch's caching allocator over this leg; "
                    "their sum bounds the leg's peak"},
    }


def psr_band(primary, horizons, vectors, mask, tile):
    """The device PSR mask of one tile against the oracle's (the reference's
    FP64 PSR on the same reduced vectors): pixels that differ, the pixels of
    the 1e-4 deg band around the limb threshold, and differences outside it."""
    from oracle import products

    tx, ty = tile
    host = horizons.cpu().numpy().reshape(TILE, TILE, AZIMUTHS)
    host = np.where(np.isneginf(host), np.float32(-50.0), host)
    started = time.perf_counter()
    expected = products.psr_tile(primary, host, vectors, tile_y=ty, tile_x=tx)
    peak = products.psr_peak_margin(primary, host, vectors, tile_y=ty, tile_x=tx)
    in_band = np.abs(peak - products.PSR_LIMB_THRESHOLD) < 1e-4
    differ = mask != expected
    return {"pixels": int(mask.size), "band_pixels": int(in_band.sum()),
            "differ": int(differ.sum()), "differ_outside_band": int((differ & ~in_band).sum()),
            "oracle_seconds": time.perf_counter() - started}


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

    # End to end through the drop-in session call with pinned host buffers,
    # over the same timed tiles as `value`: each call copies its tile's
    # segments host -> device and reads the slopes back into host memory.
    h2d = int(np.prod(segment_shape)) * 4
    d2h = TILE * TILE * AZIMUTHS * 4
    e2e_session = CudaSession(local)
    host_pyramids = [e2e_session.build_max_pyramid(dem) for dem in (primary, regional)]
    host_segments = []
    for k in range(args.warmup, total_steps):
        buffer = pinned_empty(segment_shape, np.float32)
        buffer[...] = segments[k].cpu().numpy()
        host_segments.append(buffer)

    def e2e_call(k):
        tile_row, tile_column = tiles[k]
        slopes, _ = e2e_session.subpatch_hierarchical_all_passes(
            host_segments[k - args.warmup], host_pyramids, tile_column=tile_column,
            tile_row=tile_row, tile_width=TILE, tile_height=TILE, subpatch_size=8)
        return slopes

    e2e_call(args.warmup)
    if world > 1:
        dist.barrier()
    started = time.perf_counter()
    for k in range(args.warmup, total_steps):
        e2e_call(k)
    e2e_elapsed = max_over_ranks(time.perf_counter() - started, world)
    e2e_value = world * args.steps * RAYS_PER_TILE / e2e_elapsed
    e2e_session.close()
    del host_segments

    def leg(name, run):
        """One secondary leg; on one GPU a failure is recorded in its field
        (the headline line still prints), with more ranks it propagates so
        that no rank is left waiting in a collective."""
        started = time.perf_counter()
        try:
            result = run()
        except Exception as error:
            if world > 1:
                raise
            import traceback

            traceback.print_exc()
            result = {"error": f"{type(error).__name__}: {error}"[:500]}
        log(f"[bench] {name} leg in {time.perf_counter() - started:.1f}s: "
            f"{json.dumps(result)[:2000]}")
        return result

    parity = None
    if rank == 0 and world == 1 and not args.skip_cpu:
        parity = leg("parity", lambda: site_parity(session, dems, primary, regional,
                                                    segments[args.warmup], tiles[args.warmup]))
    numba_reference = None
    if rank == 0 and world == 1 and not args.skip_reference_numba:
        tile_row, tile_column = tiles[args.warmup]
        step(args.warmup)
        torch.cuda.synchronize()
        numba_reference = leg("reference_numba_cuda", lambda: reference_numba_cuda(
            primary, regional, segments[args.warmup], tiles[args.warmup],
            output.cpu().numpy()))
        numba_reference["ours_rays_per_s_device"] = value
        numba_reference["ours_rays_per_s_e2e"] = e2e_value

    lighting = leg("lightmap", lambda: lighting_benchmark(session, dems, segments, tiles,
                                                          primary, args, world, rank))
    del segments
    multisite = None if args.skip_multisite else leg(
        "multisite", lambda: multisite_benchmark(session, stream, args, world, rank))
    adjoint = None if args.skip_adjoint else leg(
        "adjoint", lambda: adjoint_benchmark(session, args, rank))
    sensitivity = (None if args.skip_sensitivity or world > 1 else leg(
        "sensitivity", lambda: sensitivity_benchmark(session, regional, args, rank)))
    # The public generator runs on device 0 (as the reference's does): 1 GPU only.
    generate = (None if args.skip_generate or world > 1 else leg(
        "generate_horizons", lambda: generate_benchmark(primary, regional, rank)))

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
                # The march is bound by instruction issue, not by FP32 FMA
                # throughput: the share of issue slots its launch keeps busy.
                "issue_slots_busy": profiled_value("march_pass_kernel_site_tile.md",
                                                   "issue_slots_busy"),
                "issue_source": "ncu smsp__issue_active.avg.pct_of_peak_sustained_active of "
                                "one pass-0 launch (profiles/march_pass_kernel_site_tile.md)",
            },
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": "rays/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "gpu_launches": 3 * args.steps,
            "clocks": clocks,
            "segment_generation_ms_per_tile": segment_seconds * 1000.0,
            "parity": parity,
            "reference_numba_cuda": numba_reference,
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


PARITY_RAYS = 20_000


def site_parity(session, dems, primary, regional, device_segments, tile):
    """Bit parity of the timed march with the FP32 oracle on PARITY_RAYS
    random rays of the first timed site-scale tile (1440 azimuths, 200 km,
    both passes), and the distance of the reference and relative FP32
    arithmetic from the FP64 restatement on the same rays."""
    import torch

    import oracle
    from lunarscout_b200.contract import PyramidArrays, map_parameters, projection_parameters
    from lunarscout_b200.cuda_backend import SiteTile

    tile_row, tile_column = tile
    out = torch.empty((TILE * TILE, AZIMUTHS), dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    # The timed call, into a fresh buffer.
    session.march_all_passes_device(device_segments.data_ptr(), AZIMUTHS, (TILE // 8 + 2) ** 2,
                                    dems, tile_column=tile_column, tile_row=tile_row,
                                    observer_elevation_m=OBSERVER_M, device_out=out.data_ptr())
    session.synchronize()
    timed = out.cpu().numpy()
    session.march_sites([SiteTile(tuple(dems), tile_column, tile_row, RANGE_M, OBSERVER_M)],
                        device_out=out.data_ptr(), azimuth_count=AZIMUTHS,
                        traversal="relative")
    torch.cuda.synchronize()
    relative = out.cpu().numpy()
    segments = device_segments.cpu().numpy()
    pyramids = []
    for dem in (primary, regional):
        mips, levels = oracle.build_pyramid(dem.elevation_m)
        pyramids.append(PyramidArrays(dem.elevation_m, mips, levels, map_parameters(dem),
                                      projection_parameters(dem)))
    rng = np.random.default_rng(2024)
    pixels = rng.integers(0, TILE * TILE, PARITY_RAYS).astype(np.int32)
    azimuths = rng.integers(0, AZIMUTHS, PARITY_RAYS).astype(np.int32)
    common = dict(tile_column=tile_column, tile_row=tile_row, observer_elevation_m=OBSERVER_M,
                  pixels=pixels, azimuths=azimuths)
    fp32, _ = oracle.march_all_passes(segments, pyramids, **common)
    fp32_relative, _ = oracle.march_all_passes(
        segments, pyramids, mask=oracle.PRODUCTION_MASK | oracle.OPT_RELATIVE, **common)
    fp64, _ = oracle.march_all_passes(segments, pyramids, precision="f64", **common)
    got = timed[pixels, azimuths]
    got_relative = relative[pixels, azimuths]
    reference = np.degrees(np.arctan(fp64))

    def distance(values):
        d = np.abs(np.degrees(np.arctan(values.astype(np.float64))) - reference)
        d = d[np.isfinite(reference)]
        return {"p99.9": float(np.quantile(d, 0.999)), "max": float(d.max()),
                "over_0.01": int((d > 0.01).sum())}

    return {
        "workload": "first timed site-scale tile, 1440 az, 200 km, both passes",
        "rays": PARITY_RAYS,
        "c2_bits_equal": bool(np.array_equal(got, fp32)),
        "c2_relative_bits_equal": bool(np.array_equal(got_relative, fp32_relative)),
        "error_vs_fp64_deg": {"reference_arithmetic": distance(got),
                              "relative_arithmetic": distance(got_relative)},
    }


def reference_runtime():
    """The reference installed under baseline/_ref (None when absent)."""
    sys.path.insert(0, str(ROOT / "baseline"))
    import load_reference

    return load_reference if load_reference.available() else None


def reference_dem(ours):
    """This project's DemGrid as the reference's own DemGrid."""
    from lunarscout._numba_horizon import geometry

    return geometry.DemGrid(np.ascontiguousarray(ours.elevation_m, dtype=np.float32),
                            np.array(ours.geo_transform, dtype=np.float64),
                            geometry.ProjectionParameters.from_array(ours.projection.as_array()))


def reference_numba_cuda(primary, regional, device_segments, tile, ours_slopes, repeats=2):
    """The reference's own Numba-CUDA march (cuda_backend.CudaSession.
    subpatch_hierarchical_all_passes, cuda_backend.py:1445-1552) on the same
    B200, the same site-scale tile and the same segments as the timed march:
    its rays/s through that drop-in call (host segments in, host slopes out)
    and from its own per-pass CUDA-event times, and its slopes against ours."""
    runtime = reference_runtime()
    if runtime is None:
        return {"available": False, "reason": "reference not installed under baseline/_ref"}
    try:
        runtime.import_reference(enable_numba_cuda=True)
        from lunarscout._numba_horizon import cuda_backend

        session = cuda_backend.CudaSession(device_id=0)
        pyramids = [session.build_max_pyramid(reference_dem(d)) for d in (primary, regional)]
        values = device_segments.cpu().numpy()
        tile_row, tile_column = tile
        kwargs = dict(tile_column=tile_column, tile_row=tile_row, tile_width=TILE,
                      tile_height=TILE, subpatch_size=8, observer_elevation_m=OBSERVER_M)
        started = time.perf_counter()
        slopes, _ = session.subpatch_hierarchical_all_passes(values, pyramids, **kwargs)
        first_call_s = time.perf_counter() - started
        walls, kernels = [], []
        for _ in range(repeats):
            started = time.perf_counter()
            slopes, pass_seconds = session.subpatch_hierarchical_all_passes(values, pyramids,
                                                                             **kwargs)
            walls.append(time.perf_counter() - started)
            kernels.append(float(sum(pass_seconds)))
    except Exception as error:  # the JIT or the device refused: record why
        return {"available": False, "reason": f"{type(error).__name__}: {error}"[:400]}
    theirs = np.degrees(np.arctan(np.asarray(slopes, dtype=np.float64)))
    ours = np.degrees(np.arctan(np.asarray(ours_slopes, dtype=np.float64)))
    finite = np.isfinite(theirs) & np.isfinite(ours)
    wall, kernel = min(walls), min(kernels)
    return {
        "available": True,
        "how": "numba's built-in CUDA target in place of the numba-cuda package "
               "(lunarscout/_cuda_runtime.py:12 gate replaced), unmodified kernels",
        "rays_per_s_call": RAYS_PER_TILE / wall,
        "rays_per_s_kernel_events": RAYS_PER_TILE / kernel,
        "call_seconds": wall, "kernel_seconds": kernel,
        "first_call_seconds_with_jit": first_call_s,
        "slopes_bits_equal_fraction": float(np.mean(np.asarray(slopes) == ours_slopes)),
        "max_abs_deg_vs_ours": float(np.abs(theirs - ours)[finite].max()),
        "same_inf_rays": bool(np.array_equal(np.isinf(theirs), np.isinf(ours))),
    }


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
    """Four tiles of the multi-site batch through the persistent march: the
    reference traversal, the skip ladder, then the skip ladder in the
    relative arithmetic (march_sites_kernel launches 0, 1, 2); used under
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
    for traversal in ("exact", "ladder", "relative-ladder"):
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
    parser.add_argument("--skip-reference-numba", action="store_true",
                        help="leave out the reference's own Numba-CUDA march on the same tile")
    parser.add_argument("--profile", nargs="?", const="site", choices=("site", "multisite"),
                        help="small profiling case, no timing: 'site' = one site-scale tile "
                             "(two march steps, two lighting launches); 'multisite' = four "
                             "tiles through the persistent march (exact, ladder, relative ladder)")
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
