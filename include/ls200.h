/*
 * ls200 — C ABI of the B200-native lunarscout horizon-and-lighting hot path.
 *
 * Every entry point returns an ls200_status; on failure a message is kept per
 * calling thread (ls200_last_error).  No C++ exception crosses this boundary.
 * Host pointers are plain C arrays in the reference's layouts; "_device"
 * entry points take device pointers and a cudaStream_t passed as void*.
 * Calls on one context are serialised by the context's own lock, so a
 * context may be shared between threads; the GIL is released by ctypes.
 *
 * Each entry point names the reference interface it replaces
 * (paths within Costigan/lunarscout).
 */
#ifndef LS200_H
#define LS200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    LS200_OK = 0,
    LS200_ERR_INVALID = 1,     /* input contract violated (Python: ValueError) */
    LS200_ERR_CUDA = 2,        /* CUDA runtime failure during execution */
    LS200_ERR_UNAVAILABLE = 3, /* no usable sm_100 device (CudaBackendError) */
    LS200_ERR_TIMEOUT = 4,     /* a bounded device wait gave up */
} ls200_status;

typedef struct ls200_context ls200_context;
typedef struct ls200_dem ls200_dem;

/* Message of the last failed call made by this thread ("" if none). */
const char *ls200_last_error(void);
/* Library/ABI version, e.g. 1. */
int ls200_abi_version(void);

/* ---- context: src/lunarscout/_numba_horizon/cuda_backend.py:1157-1196
 *      (CudaSession.__init__, .info) ---- */
ls200_status ls200_context_create(int device_id, ls200_context **out);
ls200_status ls200_context_destroy(ls200_context *ctx);
ls200_status ls200_device_info(ls200_context *ctx, char *name, int name_capacity,
                               int *major, int *minor, int *sm_count);
/* Use `stream` (a cudaStream_t; NULL is the legacy default stream) for all
 * later work of this context. */
ls200_status ls200_set_stream(ls200_context *ctx, void *stream);
/* Go back to the context's own non-blocking stream. */
ls200_status ls200_reset_stream(ls200_context *ctx);
ls200_status ls200_synchronize(ls200_context *ctx);

/* ---- max pyramid: src/lunarscout/_numba_horizon/pyramid.py:19-31
 *      (_level_layout) and cuda_backend.py:1260-1281 (build_max_pyramid) ---- */
/* Writes up to `capacity` rows of (level, offset, width, height); returns the
 * level count through *level_count and the mip element count. */
ls200_status ls200_pyramid_layout(int width, int height, int32_t *levels, int capacity,
                                  int *level_count, int64_t *mip_count);
/* host level0 [height, width] -> host mips [mip_count] */
ls200_status ls200_build_max_pyramid(ls200_context *ctx, const float *level0, int width,
                                     int height, float *mips);

/* ---- device-resident DEM (pyramid + georeference):
 *      cuda_backend.py:1231-1258 (_prepare_production_pyramids) ---- */
/* Uploads level0 and, if `mips` is NULL, builds the pyramid on the device.
 * geo_transform: GDAL order (6 f64).  projection: radius, lat0, lon0, scale,
 * false_easting, false_northing (6 f64).  map_parameters: the reference's 11
 * float32 map parameters (pyramid.py:84-95). */
ls200_status ls200_dem_create(ls200_context *ctx, const float *level0, int width, int height,
                              const float *mips, const double *geo_transform,
                              const double *projection, const float *map_parameters,
                              ls200_dem **out);
/* A DEM must be destroyed before its context; ls200_context_destroy releases
 * the DEMs still alive, after which their handles are invalid. */
ls200_status ls200_dem_destroy(ls200_dem *dem);
/* Copies the device mips back (e.g. to write a .pyr.bin cache). */
ls200_status ls200_dem_download_mips(ls200_dem *dem, float *mips, int64_t capacity);
/* Replace the DEM's heights from device memory (width*height float32) and
 * rebuild its pyramid on the device: the differentiable path's way of
 * marching a DEM held in a framework tensor.  No reference counterpart. */
ls200_status ls200_dem_set_heights_device(ls200_dem *dem, const float *device_heights);
/* Device address of the DEM's (raw) level-0 heights. */
ls200_status ls200_dem_level0_device(ls200_dem *dem, const float **device_level0);

/* ---- ray segments: src/lunarscout/_numba_horizon/geometry.py:575-673
 *      (build_subpatch_segments_numba) and geometry_numba.py:142-364 ---- */
/* Fills segments [azimuth_count, (tile_width/subpatch+2)^2, dem_count, 18]. */
ls200_status ls200_segments(ls200_context *ctx, ls200_dem *const *dems, int dem_count,
                            int tile_column, int tile_row, int tile_width, int azimuth_count,
                            double maximum_distance_m, double observer_elevation_m,
                            int subpatch_size, float *segments);
ls200_status ls200_segments_device(ls200_context *ctx, ls200_dem *const *dems, int dem_count,
                                   int tile_column, int tile_row, int tile_width,
                                   int azimuth_count, double maximum_distance_m,
                                   double observer_elevation_m, int subpatch_size,
                                   float *device_segments);

/* ---- horizon march: cuda_backend.py:1390-1443 (subpatch_hierarchical_pass)
 *      and :1445-1552 (subpatch_hierarchical_all_passes) ---- */
/* One pass; slopes [tile_width*tile_height, azimuth_count] pixel-major are the
 * carried input (NULL = all -inf) and the output. */
ls200_status ls200_march_pass(ls200_context *ctx, const float *segments, int azimuth_count,
                              int center_count, int dem_count, const ls200_dem *primary,
                              const ls200_dem *active, int tile_column, int tile_row,
                              int tile_width, int tile_height, int subpatch_size,
                              int pass_index, float observer_elevation_m,
                              const float *slopes_in, float *slopes_out);
/* Every pass on one resident slope buffer; pass_seconds[dem_count] receives
 * CUDA-event kernel times (may be NULL). */
ls200_status ls200_march_all_passes(ls200_context *ctx, const float *segments,
                                    int azimuth_count, int center_count, int dem_count,
                                    ls200_dem *const *dems, int tile_column, int tile_row,
                                    int tile_width, int tile_height, int subpatch_size,
                                    float observer_elevation_m, float *slopes,
                                    double *pass_seconds);
/* Device-resident variant: device_segments in, device_slopes out
 * ([P, A] pixel-major slopes, or degrees when `degrees` is non-zero);
 * pass_seconds as above (NULL skips the per-pass events and the wait).
 * The host-segment entry points refuse segments on which the FP32 path
 * position would stop moving (s_end of 2048 km or more, or a pixel too small
 * for the ray length: the reference's kernel would never end there either);
 * ls200_segments_device refuses the same through its distance limit.  Device
 * segments given here are not read back: they must come from
 * ls200_segments_device or satisfy the same limits. */
ls200_status ls200_march_all_passes_device(ls200_context *ctx, const float *device_segments,
                                           int azimuth_count, int center_count,
                                           int dem_count, ls200_dem *const *dems,
                                           int tile_column, int tile_row, int tile_width,
                                           int tile_height, int subpatch_size,
                                           float observer_elevation_m, float *device_out,
                                           int degrees, double *pass_seconds);
/* Node visits (inner hierarchy iterations), level-0 samples and ray steps
 * (outer iterations) counted by the last march call of this context, when
 * counting was enabled with ls200_set_counting (a slower diagnostic build of
 * the kernel runs meanwhile). */
ls200_status ls200_set_counting(ls200_context *ctx, int enabled);
ls200_status ls200_last_counters(ls200_context *ctx, int64_t *visits, int64_t *samples,
                                 int64_t *steps);

/* One horizon tile end to end on the device, the work of one patch of
 * src/lunarscout/horizon.py:137-238 (_run_horizon_pipeline: prepare =
 * build_subpatch_segments_numba, process = generate_patch_horizons, finalize
 * = HorizonBuffers.degrees, then the .cbin encoder): segments, every DEM
 * pass, degrees, and with `compress` the .cbin payload.  Pixels outside the
 * primary DEM (partial right/bottom tiles) hold -50 degrees, as the
 * reference's writer pads them (file_format.py:93-120).  `out` (host) gets
 * the payload (capacity >= 16384*2882) or raw pixel-major float32 degrees
 * (capacity >= 16384*azimuth_count*4); *size the byte count. */
ls200_status ls200_horizon_tile(ls200_context *ctx, ls200_dem *const *dems, int dem_count,
                                int tile_column, int tile_row, int azimuth_count,
                                double maximum_distance_m, float observer_elevation_m,
                                int subpatch_size, int compress, void *out, int64_t capacity,
                                int64_t *size);

/* One 128x128 tile of one site in a multi-site batch. */
typedef struct ls200_site_tile {
    ls200_dem *const *dems;     /* the site's DEMs in pass order, primary first (1..8) */
    int dem_count;
    int tile_column, tile_row;  /* tile origin in primary-DEM pixels */
    double maximum_distance_m;  /* ray range (the public path uses 1,000 km) */
    float observer_elevation_m;
} ls200_site_tile;

/* Batched persistent march, no single reference counterpart: the work of
 * generate_patch_horizons (src/lunarscout/_numba_horizon/generator.py:11-40)
 * for `tile_count` tiles of any sites in one launch.  Segments are built on
 * the device per tile, then one resident grid marches every (tile, pixel,
 * azimuth) ray through all of its tile's DEM passes with work stealing.
 * traversal 0: the reference traversal, bit-identical to ls200_march_all_passes;
 * traversal 1: the skip ladder (a cull extends to the largest culled ancestor
 * cell, from 1 km on); traversals 2 and 3: 0 and 1 in the relative FP32
 * arithmetic (positions as an integer origin plus small offsets, level-0
 * heights relative to the observer's z, no rounded R + height), which stays
 * within ~1e-4 deg of the FP64 restatement of the march where the reference
 * arithmetic is off by up to ~0.02 deg at near-field samples.  `device_out` holds tile_count x 16384 x azimuth_count
 * floats, pixel-major per tile: slopes, or degrees when `degrees` (-inf kept
 * outside the primary DEM).  `seconds` (may be NULL) gets
 * {segments + setup, march}. */
ls200_status ls200_march_sites(ls200_context *ctx, const ls200_site_tile *tiles, int tile_count,
                               int azimuth_count, int subpatch_size, int traversal,
                               int degrees, void *device_out, double *seconds);

/* Launch configuration of ls200_march_sites for this context (results do
 * not depend on it): `lanes_per_azimuth` = how many adjacent pixels of one
 * azimuth a 32-ray warp job holds (a power of two from 1 to 32; the job then
 * spans 32 / lanes_per_azimuth azimuths), `min_blocks` = resident 128-thread blocks per SM, 8 (64
 * registers) or 6 (80 registers).  Chosen by the autotuner; defaults 2, 8. */
ls200_status ls200_set_batch_config(ls200_context *ctx, int lanes_per_azimuth, int min_blocks);
ls200_status ls200_get_batch_config(ls200_context *ctx, int *lanes_per_azimuth, int *min_blocks);

/* slope -> degrees, float32(atan(s) * float32(180/pi)), -inf preserved:
 * src/lunarscout/_numba_horizon/contract.py:362-371 (HorizonBuffers.degrees) */
ls200_status ls200_slopes_to_degrees(ls200_context *ctx, const float *slopes, int64_t count,
                                     float *degrees);

/* ---- horizon tile codec (.cbin): src/lunarscout/_numba_horizon/file_format.py:39-73
 *      (_encode_horizons_python) and :135-182 (_decode_compressed_payload_into_python) ---- */
/* Pixel-major degrees float32[16384*1440] (host) -> payload (host, capacity
 * >= 16384*2882 bytes); *size receives the payload length. */
ls200_status ls200_cbin_encode(ls200_context *ctx, const float *degrees, uint8_t *payload,
                               int64_t capacity, int64_t *size);
/* The same on device buffers (payload capacity >= 16384*2882 bytes). */
ls200_status ls200_cbin_encode_device(ls200_context *ctx, const float *device_degrees,
                                      uint8_t *device_payload, int64_t *size);
/* Payload (host) -> degrees float32[16384*1440] (host); LS200_ERR_INVALID for
 * a structurally invalid payload. */
ls200_status ls200_cbin_decode(ls200_context *ctx, const uint8_t *payload, int64_t size,
                               float *degrees);

/* ---- lighting products: src/lunarscout/_numba_horizon/lightmap_cuda.py:187-276
 *      (LightmapCudaSession) and psr_cuda.py:191-375 (PsrCudaSession) ---- */
typedef struct ls200_vectors ls200_vectors;
/* Device-resident float32 Moon-ME vectors [count, 3] (metres); the sessions
 * keep one resident per vector set (lightmap_cuda.py:238-242). */
ls200_status ls200_vectors_create(ls200_context *ctx, const float *vectors, int count,
                                  ls200_vectors **out);
ls200_status ls200_vectors_destroy(ls200_vectors *vectors);
/* Stage one 128x128 patch: patch_dem float32[128*128] (zero outside the valid
 * rect), horizons float32[128*128*1440] degrees, the DEM's geotransform and
 * projection (6 f64 each) and the patch window. */
ls200_status ls200_lighting_load(ls200_context *ctx, const float *patch_dem,
                                 const double *geo_transform, const double *projection,
                                 const float *horizons, int tile_x, int tile_y,
                                 int valid_width, int valid_height);
/* Times [time_start, time_start+time_count) of the staged patch into host
 * `out` [time_count, 128, 128]: signal 0 = float32 sun fraction, 1 = uint8
 * int(255*fraction), 2 = float32 body-centre margin (deg). */
ls200_status ls200_lighting_run(ls200_context *ctx, const ls200_vectors *vectors,
                                int time_start, int time_count, int signal, void *out);
/* PSR byte mask (255 = permanently shadowed) of the staged patch over all
 * vectors into host out[128*128]. */
ls200_status ls200_psr_run(ls200_context *ctx, const ls200_vectors *vectors, uint8_t *out);
/* The PSR vector reduction, replacing reduce_sun_vectors_for_psr
 * (src/lunarscout/_numba_horizon/psr.py:61-91, called once per product at
 * psr_pipeline.py:259-263): for the DEM's four corner pixels and its centre
 * pixel and 1440 azimuth bins of 0.25 deg, the index of the highest vector
 * (first on ties), listed viewpoint by viewpoint, bin by bin, each index once
 * in order of first appearance.  FP64 on the device.  dem: host float32
 * [height, width] (only the five viewpoints' elevations are read);
 * vectors: host float64 [count, 3] Moon-ME metres; indices_out: room for
 * 7200 int64; *reduced_count receives how many were written.  Synchronous. */
ls200_status ls200_psr_reduce_vectors(ls200_context *ctx, const float *dem, int width,
                                      int height, const double *geo_transform,
                                      const double *projection, const double *vectors,
                                      int count, int64_t *indices_out, int *reduced_count);
/* Device-resident batch of up to 32 patches: device patch_dems
 * [n,128,128], host geo_transforms/projections [n,6] f64, host windows
 * [n,4] (tile_x, tile_y, valid_width, valid_height), device horizons
 * [n,128,128,1440], device frames scratch [n,16384,12] f32, device out
 * [n, time_count, 128*128] (PSR, signal 3: [n, 128*128] over all vectors).
 * Steps are evaluated in the table's longitude order (outputs stay in time
 * order).  A launch over part of the table first writes that part of the
 * order into a buffer the table owns, so launches on one table that may run
 * at the same time on different streams race on it; on the context's own
 * stream they are ordered. */
ls200_status ls200_lighting_device(ls200_context *ctx, int tile_count, const float *patch_dems,
                                   const double *geo_transforms, const double *projections,
                                   const int32_t *windows, const float *horizons,
                                   const ls200_vectors *vectors, int time_start,
                                   int time_count, int signal, float *frames, void *out);
/* Allocation-free twin of ls200_lighting_device, for callers that may not
 * call cudaMalloc when they run (their device memory belongs to another
 * allocator, or they cannot afford an allocation's device-wide
 * synchronisation).  No counterpart in the reference.  Inputs and outputs
 * are the caller's device buffers (vectors: float32[vector_count, 3]); the
 * per-pixel frame scratch is a fixed 3 MiB device array inside this library,
 * so tile_count is at most 4 and larger batches are rejected with
 * LS200_ERR_INVALID.  The first call on a device looks up that array's
 * address and uploads the disk constants; make it before any stream capture.
 * All calls share the array: calls that overlap on the GPU (two streams, two
 * contexts on one device) race on it.  Nothing in it needs to start at zero.
 * The array's address is cached per device index; after cudaDeviceReset the
 * library must be reloaded before this entry point is called again.  It takes
 * the table as plain vectors with no longitude order, so it evaluates steps in
 * time order: the same products as ls200_lighting_device, but slower on long
 * tables (a year hourly: about 0.4x its throughput).
 * Runs asynchronously on the context's stream. */
ls200_status ls200_lighting_device_noalloc(ls200_context *ctx, int tile_count,
                                           const float *patch_dems,
                                           const double *geo_transforms,
                                           const double *projections, const int32_t *windows,
                                           const float *horizons, const float *device_vectors,
                                           int vector_count, int time_start, int time_count,
                                           int signal, void *out);
/* ---- CUDA graphs of asynchronous device calls (no reference counterpart;
 *      replaces the per-chunk launch-and-wait loop of
 *      src/lunarscout/_numba_horizon/lightmap_cuda.py:226-276) ----
 * Between ls200_capture_begin and ls200_capture_end the context's stream
 * records instead of running: asynchronous entry points (ls200_lighting_device
 * over its time chunks, the *_device march / segment entries) become graph
 * nodes bound to the device buffers they were given.  ls200_graph_launch
 * replays the whole graph with one launch on the context's stream; buffer
 * contents may change between launches.  A call that waits for the host
 * inside a capture fails and invalidates it (ls200_capture_end then returns
 * an error).  The context must use a created stream (not NULL).  Destroy
 * graphs before their context. */
typedef struct ls200_graph ls200_graph;
ls200_status ls200_capture_begin(ls200_context *ctx);
ls200_status ls200_capture_end(ls200_context *ctx, ls200_graph **out);
ls200_status ls200_graph_launch(ls200_graph *graph);
ls200_status ls200_graph_nodes(ls200_graph *graph, int64_t *nodes);
ls200_status ls200_graph_destroy(ls200_graph *graph);

/* ---- mission duration: src/lunarscout/_numba_horizon/mission_duration.py:
 *      164-256 (reduce_longest_candidate_duration_stream) over the condition
 *      of mission_duration_pipeline.py:88-349 (fraction >= threshold, and
 *      with Earth vectors Earth margin >= threshold), fused with the
 *      lightmap so the condition stream is never materialised ----
 * Tiles as in ls200_lighting_device (device patch DEMs and horizons, host
 * geotransforms / projections / windows); sun (and optional earth) vector
 * tables of the same length T; sample_hours (host f64[T]) the duration
 * credited to each sample; start_windows (host int32[I][2]) the (first, end)
 * sample indices of each candidate start window, I <= 64.  out (device)
 * float32 [tiles, I, 16384]: the longest right-censored run per window, in
 * hours or, with output_days, days. */
ls200_status ls200_mission_duration_device(
    ls200_context *ctx, int tile_count, const float *patch_dems, const double *geo_transforms,
    const double *projections, const int32_t *windows, const float *horizons,
    const ls200_vectors *sun, const ls200_vectors *earth, float sun_threshold,
    float earth_threshold, const double *sample_hours, const int32_t *start_windows,
    int interval_count, int output_days, float *out);

/* ---- safe haven: src/lunarscout/_numba_horizon/safe_haven.py:75-243
 *      (reduce_safe_haven_patch_stream) over the fraction and Earth-margin
 *      streams that safe_haven_pipeline.py:240-272 feeds it, fused with the
 *      lightmap so neither stream is materialised ----
 * Tiles as in ls200_lighting_device; sun and earth vector tables of the same
 * length T; month_index_of (host int32[T]) the month band of each time step
 * (-1 for none, else < band_count).  Low Sun is fraction < sunlight_threshold
 * (in [0, 1]); an Earth outage is margin < earth_threshold_deg (finite).
 * out (device) float32 [tiles, band_count, 16384]: per band the longest
 * low-Sun run that overlapped an outage within the band, times
 * time_step_hours (> 0); NaN where the band saw no outage or only outages,
 * and outside each tile's valid rectangle. */
ls200_status ls200_safe_haven_device(
    ls200_context *ctx, int tile_count, const float *patch_dems, const double *geo_transforms,
    const double *projections, const int32_t *windows, const float *horizons,
    const ls200_vectors *sun, const ls200_vectors *earth, float sunlight_threshold,
    float earth_threshold_deg, float time_step_hours, const int32_t *month_index_of,
    int band_count, float *out);
/* ---- Earth-visibility fraction: mean over time of (Earth margin >=
 *      threshold), the margin being iter_patch_margin_tiles'
 *      (src/lunarscout/_numba_horizon/lightmap_cuda.py:125-145,
 *      lightmap_cpu.py:121-141) for the Earth vectors ----
 * Tiles as in ls200_lighting_device; earth: vector table of T steps.  out
 * (device) float32 [tiles, 16384]: count / T per pixel (FP64 division rounded
 * to float32), NaN outside each tile's valid rectangle. */
ls200_status ls200_earth_visibility_device(ls200_context *ctx, int tile_count,
                                           const float *patch_dems,
                                           const double *geo_transforms,
                                           const double *projections, const int32_t *windows,
                                           const float *horizons, const ls200_vectors *earth,
                                           float threshold_deg, float *out);
/* Diagnostic: sun fraction at given (azimuth, elevation) in degrees for n
 * horizon rows float32[n,1440] (lightmap.py:32-73). */
ls200_status ls200_sun_fraction(ls200_context *ctx, const float *horizons,
                                const float *azimuth_deg, const float *elevation_deg, int n,
                                float *out);

/* ---- host memory: src/lunarscout/_numba_horizon/psr_cuda.py:234-238
 *      (allocate_pinned_horizon_buffer) ---- */
/* Page-locked host memory for H2D/D2H staging (cudaHostAlloc). */
ls200_status ls200_host_alloc(int64_t bytes, void **out);
ls200_status ls200_host_free(void *ptr);

/* ---- DEM adjoint of a time-integrated sun fraction (no reference
 *      counterpart; the interpolation of the horizon at the sun azimuth is
 *      nh/lightmap_cuda.py:125-145's) ----
 * loss = sum over tiles, pixels of w * mean over the `sun` vectors of
 * F((el - h) / r): F = visible fraction of a disk of radius r (degrees)
 * above a level horizon line, h = the horizon (degrees, clamped at -90)
 * interpolated at the sun azimuth.  Every tile must use the same DEM stack.
 * The forward marches the tiles (ls200_march_sites, `traversal` 0 or 1) with
 * one checkpoint per ray (the winning sample) kept in the context for the
 * next backward; device_weights holds tile_count x 16384 float32.  seconds
 * (may be NULL) gets {march, lighting + loss}.  The backward adds
 * grad_output * dloss/dheight into device_grads[d] (float64 [H_d, W_d], one
 * per DEM of the stack, accumulated); *seconds (may be NULL) its time. */
ls200_status ls200_sun_loss_forward(ls200_context *ctx, const ls200_site_tile *tiles,
                                    int tile_count, int azimuth_count, int traversal,
                                    const float *device_weights, const ls200_vectors *sun,
                                    double disk_radius_deg, double *loss, double *seconds);
ls200_status ls200_sun_loss_backward(ls200_context *ctx, double grad_output,
                                     double *const *device_grads, int grad_count,
                                     double *seconds);
/* The last forward's loss re-evaluated at the DEMs' current heights with its
 * sampling held fixed: every ray's horizon is recomputed (FP64) from its
 * recorded winning sample.  A following backward differentiates this
 * function, whose finite differences then match the adjoint. */
ls200_status ls200_sun_loss_replay(ls200_context *ctx, double *loss);
/* Host copies of the last forward's checkpoints (rays x 4 float: px, py,
 * distance m, slope; flags = pass << 1 | near, 0xff for none), sun
 * directions ([tiles, T, 16384] x (azimuth, elevation) degrees) and horizons
 * (degrees); any pointer may be NULL. */
ls200_status ls200_sun_loss_checkpoints(ls200_context *ctx, float *points, uint8_t *flags,
                                        float *directions, float *horizons);

/* FP32 FMA issue-rate probe (TFLOP/s, 2 flops per FMA) on this device: the
 * measured denominator of the march's FP32 roofline.  No reference
 * counterpart. */
ls200_status ls200_fp32_probe(ls200_context *ctx, int iterations, double *tflops);

/* Exhaustive check of the march's correctly rounded reciprocal (a hardware
 * approximation plus one Newton-Raphson correction) against the IEEE
 * round-to-nearest reciprocal on this device, over every 32-bit pattern with
 * |x| >= 2^-64, both signs: `mismatches` = results that differ in any bit
 * (must be 0), `checked` = results compared.  No reference counterpart. */
ls200_status ls200_check_arithmetic(ls200_context *ctx, int64_t *mismatches, int64_t *checked);

/* Device memory held by this library's own allocations on `device` (DEMs,
 * vector tables, context buffers; not the caller's buffers): bytes in use now
 * and the high-water mark since load or the last reset; reset_peak != 0 sets
 * the mark to the bytes in use.  Either pointer may be NULL.  No reference
 * counterpart (the reference reports cudaMemGetInfo snapshots). */
ls200_status ls200_memory_stats(int device, int64_t *in_use, int64_t *peak, int reset_peak);

#ifdef __cplusplus
}
#endif

#endif /* LS200_H */
