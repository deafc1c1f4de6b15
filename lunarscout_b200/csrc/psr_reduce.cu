// The PSR vector reduction on the device (src/lunarscout/_numba_horizon/
// psr.py:61-91, reduce_sun_vectors_for_psr): for five viewpoints of the DEM
// (its four corner pixels and its centre pixel) and 1440 azimuth bins of
// 0.25 deg, keep the vector with the highest elevation seen from that
// viewpoint in that bin (the first one on ties), then list the kept vector
// indices viewpoint by viewpoint, bin by bin, each index once, in the order
// of its first appearance.  The PSR pipeline evaluates the patches against
// the reduced vectors only (psr_pipeline.py:259-263).
//
// Arithmetic: FP64, as the reference (psr.py:29-58): the viewpoint's east /
// north / up frame from the stereographic inverse, the vector rotated into
// it and translated by -(R + h) up, azimuth = atan2(e, n) in degrees wrapped
// to [0, 360), elevation = atan2(u, hypot(e, n)) in degrees.  Every product
// and sum rounds separately (the library builds with --fmad=false).
//
// Kernels: (1) one thread per (viewpoint, vector) computes the azimuth bin
// and the elevation and raises the bin's maximum with a 64-bit atomicMax on
// an order-preserving integer image of the elevation; (2) the threads whose
// elevation equals their bin's maximum take the bin with atomicMin on the
// vector index (first on ties); (3) each kept index records its first
// position in the viewpoint-major bin list with atomicMin; (4) one block
// keeps the first positions and compacts them in order with a block scan.
#include <algorithm>

#include "internal.cuh"

namespace ls200 {

constexpr int kViewpoints = 5;
constexpr int kBins = 1440;
constexpr int kBinSlots = kViewpoints * kBins;  // 7200
constexpr int kNone = 0x7f7f7f7f;                // memset(0x7f) sentinel, > any index

struct ViewpointSet {
    int row[kViewpoints], column[kViewpoints];
    double height[kViewpoints];  // DEM elevation at the viewpoint (float32 widened)
    double gt[6], proj[6];
};

// Order-preserving map of a double to an unsigned integer; NaN maps to 0,
// below every number.
__device__ __forceinline__ unsigned long long order_key(double value) {
    if (value != value) return 0ull;
    const unsigned long long bits = static_cast<unsigned long long>(__double_as_longlong(value));
    return (bits >> 63) ? ~bits : (bits | 0x8000000000000000ull);
}

// East/north/up rotation (columns) and translation of one viewpoint
// (psr.py:29-48 with geometry.py:85-90, 153-174).
__device__ void viewpoint_frame(const ViewpointSet &V, int p, double rot[3][3], double trans[3]) {
    const double *gt = V.gt, *proj = V.proj;
    const double column = V.column[p], row = V.row[p];
    const double crs_x = gt[0] + gt[1] * column + gt[2] * row;
    const double crs_y = gt[3] + gt[4] * column + gt[5] * row;
    const double xp = crs_x - proj[4], yp = crs_y - proj[5];
    const double rho = hypot(xp, yp);
    double latitude, longitude;
    if (rho < 1e-9) {
        latitude = proj[1];
        longitude = proj[2];
    } else {
        const double c = 2.0 * atan2(rho, 2.0 * proj[3] * proj[0]);
        const double sin_c = sin(c), cos_c = cos(c);
        const double sin_o = sin(proj[1]), cos_o = cos(proj[1]);
        latitude = asin(cos_c * sin_o + yp * sin_c * cos_o / rho);
        longitude = proj[2] + atan2(xp * sin_c, rho * cos_o * cos_c - yp * sin_o * sin_c);
    }
    const double cos_lat = cos(latitude), sin_lat = sin(latitude);
    const double cos_lon = cos(longitude), sin_lon = sin(longitude);
    const double up[3] = {cos_lat * cos_lon, cos_lat * sin_lon, sin_lat};
    const double east[3] = {-sin_lon, cos_lon, 0.0};
    const double north[3] = {-sin_lat * cos_lon, -sin_lat * sin_lon, cos_lat};
    const double radius = proj[0] + V.height[p];
    for (int k = 0; k < 3; ++k) {
        rot[k][0] = east[k];
        rot[k][1] = north[k];
        rot[k][2] = up[k];
    }
    for (int j = 0; j < 3; ++j)
        trans[j] = -(radius * up[0] * rot[0][j] + radius * up[1] * rot[1][j] +
                     radius * up[2] * rot[2][j]);
}

// Kernel 1: grid (vector blocks, viewpoints).
__global__ void viewpoint_bins_kernel(const __grid_constant__ ViewpointSet V,
                                      const double *__restrict__ vectors, int count,
                                      unsigned long long *__restrict__ keys,
                                      int *__restrict__ bins,
                                      unsigned long long *__restrict__ maxima) {
    __shared__ double frame[12];
    const int p = blockIdx.y;
    if (threadIdx.x == 0) {
        double rot[3][3], trans[3];
        viewpoint_frame(V, p, rot, trans);
        for (int k = 0; k < 9; ++k) frame[k] = rot[k / 3][k % 3];
        for (int j = 0; j < 3; ++j) frame[9 + j] = trans[j];
    }
    __syncthreads();
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < count; t += gridDim.x * blockDim.x) {
        const size_t v = 3 * static_cast<size_t>(t);
        const double v0 = vectors[v], v1 = vectors[v + 1], v2 = vectors[v + 2];
        double e[3];
        for (int j = 0; j < 3; ++j)
            e[j] = v0 * frame[j] + v1 * frame[3 + j] + v2 * frame[6 + j] + frame[9 + j];
        double azimuth = atan2(e[0], e[1]) * (180.0 / 3.141592653589793);
        azimuth = fmod(azimuth, 360.0);
        if (azimuth < 0.0) azimuth += 360.0;
        const double elevation = atan2(e[2], hypot(e[0], e[1])) * (180.0 / 3.141592653589793);
        const double scaled = azimuth * (static_cast<double>(kBins) / 360.0);
        // NaN or out-of-range azimuths cannot win a bin (their elevation is
        // NaN too, which never compares greater); park them on bin 0 unkeyed.
        int bin = 0;
        unsigned long long key = 0ull;
        if (scaled >= 0.0 && scaled < 2.0 * kBins) {
            bin = static_cast<int>(static_cast<long long>(scaled) % kBins);
            key = order_key(elevation);
        }
        const size_t slot = static_cast<size_t>(p) * count + t;
        keys[slot] = key;
        bins[slot] = bin;
        if (key) atomicMax(maxima + p * kBins + bin, key);
    }
}

// Kernel 2: the first vector reaching its bin's maximum takes the bin.
__global__ void select_bins_kernel(const unsigned long long *__restrict__ keys,
                                   const int *__restrict__ bins, int count,
                                   const unsigned long long *__restrict__ maxima,
                                   int *__restrict__ selected) {
    const long long total = static_cast<long long>(kViewpoints) * count;
    for (long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; i < total;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const int p = static_cast<int>(i / count);
        const int t = static_cast<int>(i - static_cast<long long>(p) * count);
        const unsigned long long key = keys[i];
        const int slot = p * kBins + bins[i];
        if (key && key == maxima[slot]) atomicMin(selected + slot, t);
    }
}

// Kernel 3: first position of each kept index in the viewpoint-major list.
__global__ void first_position_kernel(const int *__restrict__ selected,
                                      int *__restrict__ first) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < kBinSlots && selected[i] != kNone) atomicMin(first + selected[i], i);
}

// Kernel 4 (one block of 1024 threads): keep each index at its first
// position and write the kept indices in list order.
__global__ void __launch_bounds__(1024) compact_kernel(const int *__restrict__ selected,
                                                       const int *__restrict__ first,
                                                       int *__restrict__ out,
                                                       int *__restrict__ out_count) {
    constexpr int kPer = (kBinSlots + 1023) / 1024;  // 8 slots per thread
    __shared__ int sums[1024];
    const int base = threadIdx.x * kPer;
    int keep[kPer];
    int local = 0;
#pragma unroll
    for (int k = 0; k < kPer; ++k) {
        const int i = base + k;
        const int v = i < kBinSlots ? selected[i] : kNone;
        keep[k] = (v != kNone && first[v] == i) ? 1 : 0;
        local += keep[k];
    }
    sums[threadIdx.x] = local;
    __syncthreads();
    // Inclusive Hillis-Steele scan over the 1024 thread sums.
    for (int offset = 1; offset < 1024; offset <<= 1) {
        const int add = threadIdx.x >= offset ? sums[threadIdx.x - offset] : 0;
        __syncthreads();
        sums[threadIdx.x] += add;
        __syncthreads();
    }
    int position = sums[threadIdx.x] - local;
#pragma unroll
    for (int k = 0; k < kPer; ++k) {
        if (keep[k]) out[position++] = selected[base + k];
    }
    if (threadIdx.x == 1023) *out_count = sums[1023];
}

static size_t align_up(size_t n) { return (n + 255) & ~size_t(255); }

}  // namespace ls200

using namespace ls200;

extern "C" ls200_status ls200_psr_reduce_vectors(ls200_context *ctx, const float *dem, int width,
                                                 int height, const double *geo_transform,
                                                 const double *projection,
                                                 const double *vectors, int count,
                                                 int64_t *indices_out, int *reduced_count) {
    return guard([&] {
        LS_REQUIRE(ctx && dem && geo_transform && projection && vectors && indices_out &&
                       reduced_count,
                   "NULL argument");
        LS_REQUIRE(width >= 1 && height >= 1, "DEM dimensions must be positive");
        LS_REQUIRE(count >= 1 && count < (1 << 30), "vector count out of range");
        ViewpointSet V{};
        const int rows[kViewpoints] = {0, 0, height - 1, height - 1, height / 2};
        const int columns[kViewpoints] = {0, width - 1, 0, width - 1, width / 2};
        for (int p = 0; p < kViewpoints; ++p) {
            V.row[p] = rows[p];
            V.column[p] = columns[p];
            V.height[p] = static_cast<double>(dem[static_cast<size_t>(rows[p]) * width +
                                                  columns[p]]);
        }
        std::memcpy(V.gt, geo_transform, sizeof V.gt);
        std::memcpy(V.proj, projection, sizeof V.proj);

        std::lock_guard<std::mutex> hold(ctx->lock);
        activate(ctx);
        const size_t n = static_cast<size_t>(count);
        const size_t off_vectors = 0;
        const size_t off_keys = align_up(off_vectors + sizeof(double) * 3 * n);
        const size_t off_bins = align_up(off_keys + sizeof(unsigned long long) * kViewpoints * n);
        const size_t off_maxima = align_up(off_bins + sizeof(int) * kViewpoints * n);
        const size_t off_selected = align_up(off_maxima + sizeof(unsigned long long) * kBinSlots);
        const size_t off_first = align_up(off_selected + sizeof(int) * kBinSlots);
        const size_t off_out = align_up(off_first + sizeof(int) * n);
        const size_t off_count = align_up(off_out + sizeof(int) * kBinSlots);
        const size_t total = off_count + sizeof(int);
        ctx->scratch.reserve(total);
        char *base = ctx->scratch.as<char>();
        double *d_vectors = reinterpret_cast<double *>(base + off_vectors);
        auto *d_keys = reinterpret_cast<unsigned long long *>(base + off_keys);
        int *d_bins = reinterpret_cast<int *>(base + off_bins);
        auto *d_maxima = reinterpret_cast<unsigned long long *>(base + off_maxima);
        int *d_selected = reinterpret_cast<int *>(base + off_selected);
        int *d_first = reinterpret_cast<int *>(base + off_first);
        int *d_out = reinterpret_cast<int *>(base + off_out);
        int *d_count = reinterpret_cast<int *>(base + off_count);
        cudaStream_t s = ctx->stream;
        LS_CUDA(cudaMemcpyAsync(d_vectors, vectors, sizeof(double) * 3 * n,
                                cudaMemcpyHostToDevice, s));
        LS_CUDA(cudaMemsetAsync(d_maxima, 0, sizeof(unsigned long long) * kBinSlots, s));
        LS_CUDA(cudaMemsetAsync(d_selected, 0x7f, sizeof(int) * kBinSlots, s));
        LS_CUDA(cudaMemsetAsync(d_first, 0x7f, sizeof(int) * n, s));
        const int per_view = static_cast<int>(std::min<size_t>((n + 255) / 256, 1024));
        viewpoint_bins_kernel<<<dim3(per_view, kViewpoints), 256, 0, s>>>(
            V, d_vectors, count, d_keys, d_bins, d_maxima);
        LS_CUDA(cudaGetLastError());
        const int select_blocks =
            static_cast<int>(std::min<size_t>((kViewpoints * n + 255) / 256, 4096));
        select_bins_kernel<<<select_blocks, 256, 0, s>>>(d_keys, d_bins, count, d_maxima,
                                                         d_selected);
        LS_CUDA(cudaGetLastError());
        first_position_kernel<<<(kBinSlots + 255) / 256, 256, 0, s>>>(d_selected, d_first);
        LS_CUDA(cudaGetLastError());
        compact_kernel<<<1, 1024, 0, s>>>(d_selected, d_first, d_out, d_count);
        LS_CUDA(cudaGetLastError());
        int kept = 0;
        LS_CUDA(cudaMemcpyAsync(&kept, d_count, sizeof(int), cudaMemcpyDeviceToHost, s));
        LS_CUDA(cudaStreamSynchronize(s));
        LS_REQUIRE(kept >= 0 && kept <= kBinSlots, "reduction produced an invalid count");
        int host_out[kBinSlots];
        if (kept > 0) {
            LS_CUDA(cudaMemcpyAsync(host_out, d_out, sizeof(int) * kept, cudaMemcpyDeviceToHost,
                                    s));
            LS_CUDA(cudaStreamSynchronize(s));
        }
        for (int i = 0; i < kept; ++i) indices_out[i] = host_out[i];
        *reduced_count = kept;
    });
}
