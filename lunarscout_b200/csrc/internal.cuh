// Internal declarations shared by the ls200 translation units.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <set>
#include <stdexcept>
#include <string>

#include "../../include/ls200.h"

namespace ls200 {

constexpr int kMaxLevels = 20;   // 4^19 cells per side is far beyond any DEM
constexpr int kSegmentFields = 18;
constexpr int kMarchFields = 16;  // fields 0,1,4..17 of a segment

// float32(180) / float32(pi) evaluated in float32, the factor of
// HorizonBuffers.degrees (one ulp below float32(180/pi)).
constexpr float kSlopeDegrees = 0x1.ca5dcp+5f;

// An error carrying the status it maps to at the C boundary.
struct Error : std::runtime_error {
    ls200_status status;
    Error(ls200_status s, const std::string &message) : std::runtime_error(message), status(s) {}
};

void set_last_error(const std::string &message);

#define LS_CUDA(call)                                                                  \
    do {                                                                               \
        cudaError_t e_ = (call);                                                       \
        if (e_ != cudaSuccess) {                                                       \
            throw ::ls200::Error(LS200_ERR_CUDA, std::string(#call) + ": " +           \
                                                     cudaGetErrorString(e_));          \
        }                                                                              \
    } while (0)

#define LS_REQUIRE(cond, message)                                                      \
    do {                                                                               \
        if (!(cond)) throw ::ls200::Error(LS200_ERR_INVALID, (message));               \
    } while (0)

// Run `body` and translate exceptions into a status + thread-local message.
template <class F>
ls200_status guard(F &&body) {
    try {
        body();
        return LS200_OK;
    } catch (const Error &e) {
        set_last_error(e.what());
        return e.status;
    } catch (const std::bad_alloc &) {
        set_last_error("host allocation failed");
        return LS200_ERR_CUDA;
    } catch (const std::exception &e) {
        set_last_error(e.what());
        return LS200_ERR_CUDA;
    } catch (...) {
        set_last_error("unknown failure");
        return LS200_ERR_CUDA;
    }
}

// Device allocations of the library go through these two calls, which keep a
// per-device count of the bytes in use and its high-water mark
// (ls200_memory_stats).
cudaError_t tracked_malloc_bytes(void **ptr, size_t bytes);
cudaError_t tracked_free(void *ptr);
template <class T>
cudaError_t tracked_malloc(T **ptr, size_t bytes) {
    return tracked_malloc_bytes(reinterpret_cast<void **>(ptr), bytes);
}

// A growable device buffer owned by a context.
struct DeviceBuffer {
    void *ptr = nullptr;
    size_t bytes = 0;
    void reserve(size_t n) {
        if (n <= bytes) return;
        if (ptr) tracked_free(ptr);
        ptr = nullptr;
        bytes = 0;
        LS_CUDA(tracked_malloc(&ptr, n));
        bytes = n;
    }
    template <class T>
    T *as() const { return static_cast<T *>(ptr); }
    ~DeviceBuffer() {
        if (ptr) tracked_free(ptr);
    }
};

struct PyramidLevel {
    int offset, width, height;
};

struct LightingState;  // lighting tile buffers of a context (lighting_api.cu)
struct CodecBuffers;   // .cbin codec buffers of a context (codec.cu)
struct AdjointState;   // checkpoints of the last sun-loss forward (adjoint.cu)

}  // namespace ls200

struct ls200_dem {
    ls200_context *ctx = nullptr;
    int width = 0, height = 0;
    int level_count = 0;
    int64_t mip_count = 0;
    ls200::PyramidLevel levels[ls200::kMaxLevels];
    float *level0 = nullptr;  // device [height, width], as given
    // device [height*width + mip_count]: level 0 with every invalid value
    // (NaN, +-inf, <= -20000) replaced by -32000, then the packed mips.
    float *cells = nullptr;
    float *mips = nullptr;    // = cells + height*width
    // device, the layout of `cells`: each cell's four-cell bound, the maximum
    // of the cell and its right, lower and lower-right neighbours on its level
    // (-32000 for a neighbour outside the level).  The march reads one value
    // per node visit instead of four.
    float *bounds = nullptr;
    double geo_transform[6];
    double projection[6];
    float map_parameters[11];
};

struct ls200_context {
    int device = 0;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    std::mutex lock;
    cudaDeviceProp props{};
    ls200::DeviceBuffer segments;   // [A, C, D, 18]
    ls200::DeviceBuffer slopes;     // az-major working slopes [A, P]
    ls200::DeviceBuffer output;     // pixel-major [P, A]
    ls200::DeviceBuffer scratch;
    ls200::DeviceBuffer counters;   // 3 x u64: node visits, level-0 samples, ray steps
    bool counting = false;
    uint64_t last_visits = 0, last_samples = 0, last_steps = 0;
    cudaEvent_t events[ls200::kMaxLevels + 2] = {};
    std::set<ls200_dem *> dems;  // live DEMs, released with the context
    ls200::LightingState *lighting = nullptr;
    ls200::CodecBuffers *codec = nullptr;
    ls200::AdjointState *adjoint = nullptr;
    // Launch configuration of the persistent multi-site march.
    int batch_lanes_per_azimuth = 2;   // pixels of one azimuth in a 32-ray job (1..32)
    int batch_min_blocks = 8;          // resident 128-thread blocks per SM (8 or 6)
};

namespace ls200 {

// Make the context's device current on this thread.
void activate(ls200_context *ctx);

// Free the lighting buffers and vector tables owned by a context.
void release_lighting_state(ls200_context *ctx);
// Free the codec buffers owned by a context.
void release_codec(ls200_context *ctx);
// Free the adjoint checkpoints owned by a context.
void release_adjoint_state(ls200_context *ctx);
// .cbin-encode device degrees [16384, 1440] into device `payload` (capacity
// >= 16384 * 2882 bytes) on ctx->stream; returns the size (synchronises).
int64_t cbin_encode(ls200_context *ctx, const float *degrees, uint8_t *payload);

int pyramid_layout(int width, int height, PyramidLevel *levels, int capacity,
                   int64_t *mip_count);

// Build all mip levels of `dem` on ctx->stream from dem->level0.
void build_pyramid_device(ls200_context *ctx, ls200_dem *dem);
// Write the sanitized level 0 at the start of dem->cells.
void sanitize_level0(ls200_context *ctx, ls200_dem *dem);
// Write dem->bounds from dem->cells (after both parts of cells are final).
void build_cell_bounds(ls200_context *ctx, ls200_dem *dem);

// Mean pixel size (m) of a DEM from its map parameters, in FP64.
double dem_resolution_m(const ls200_dem *dem);
// Refuses a march whose rays would step in place.  The march (like the
// reference's kernel) advances its FP32 path position s (km) by at least
// 1e-4 km per cull and at least half a pixel per level-0 sample; each must
// exceed half an ulp of s, or s stops moving and the ray never ends.  Below
// 2048 km the cull advance always does; the sample advance, half a pixel of
// the active DEM, is required to exceed 2 ulp(s_end_km) (a factor four of
// margin).
void require_march_progress(double s_end_km, const ls200_dem *active);

// Segment generation into device memory.
void segments_device(ls200_context *ctx, ls200_dem *const *dems, int dem_count,
                     int tile_column, int tile_row, int tile_width, int azimuth_count,
                     double maximum_distance_m, double observer_elevation_m, int subpatch,
                     float *device_segments);

struct MarchTile {
    const float *segments;  // device [A, C, D, 18]
    int azimuth_count, center_count, dem_count;
    int tile_column, tile_row, tile_width, tile_height, subpatch;
    float observer_elevation;
};

// One pass into the az-major working buffer slopes[A, P]; first_pass starts
// every ray at -inf without reading `slopes`.
void march_pass_device(ls200_context *ctx, const MarchTile &tile, const ls200_dem *primary,
                       const ls200_dem *active, int pass_index, bool first_pass,
                       float *slopes_az_major);

// The persistent multi-site march (march_batch.cu): validates, takes the
// context lock, builds segments and marches every tile into device_out
// ([tile_count, 16384, A]); with `checkpoints` it also records each ray's
// winning sample (see SitesParams) for the DEM adjoint.
void march_sites_run(ls200_context *ctx, const ls200_site_tile *tiles, int tile_count,
                     int azimuth_count, int subpatch_size, int traversal, bool degrees,
                     float *device_out, double *seconds, float4 *checkpoints,
                     uint8_t *checkpoint_flags);

// Zero the march counters before a counted launch / read them back after it
// (both no-ops unless counting is enabled).
void reset_counters(ls200_context *ctx);
void resolve_counters(ls200_context *ctx);

// az-major [A, P] -> pixel-major [P, A], optionally as degrees.
void transpose_slopes(ls200_context *ctx, const float *az_major, int azimuth_count,
                      int pixel_count, float *pixel_major, bool degrees);
void pixel_major_to_az_major(ls200_context *ctx, const float *pixel_major, int azimuth_count,
                             int pixel_count, float *az_major);
void slopes_to_degrees_device(ls200_context *ctx, const float *slopes, int64_t count,
                              float *degrees);

}  // namespace ls200
