// Factor-four maximum-elevation pyramid (pyramid.py:19-31,110-138;
// cuda_backend.py:134-153).  Each mip cell holds the maximum valid elevation
// (finite and > -20000) of its 4x4 block of the level below, or -32000 when
// the block has no valid cell.  One launch per level, all on the context
// stream with no host round trip between levels.
#include "march_core.cuh"

namespace ls200 {

__device__ __forceinline__ bool valid_elevation(float v) {
    return !isnan(v) && !isinf(v) && v > -20000.0f;
}

// One thread per destination cell; a warp covers 32 adjacent destination
// columns, i.e. 128 contiguous source floats on each of the 4 source rows.
__global__ void __launch_bounds__(256) pyramid_downsample(const float *__restrict__ source,
                                                          int source_width, int source_height,
                                                          float *__restrict__ destination,
                                                          int width, int height) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= width || y >= height) return;
    float best = -32000.0f;
    const int x0 = x * 4, y0 = y * 4;
#pragma unroll
    for (int dy = 0; dy < 4; ++dy) {
        const int yy = y0 + dy;
        if (yy >= source_height) break;
        const float *row = source + static_cast<size_t>(yy) * source_width;
#pragma unroll
        for (int dx = 0; dx < 4; ++dx) {
            const int xx = x0 + dx;
            if (xx < source_width) {
                const float v = __ldg(row + xx);
                if (valid_elevation(v) && v > best) best = v;
            }
        }
    }
    destination[static_cast<size_t>(y) * width + x] = best;
}

// Invalid elevations become the -32000 block sentinel.  Every value the
// march then reads is either valid (> -20000, finite) or exactly -32000, so
// validity is one comparison and a four-cell bound is a plain maximum with
// the same result as the reference's filtered maximum.
__global__ void sanitize_kernel(const float *__restrict__ in, long long n,
                                float *__restrict__ out) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const float v = in[i];
        out[i] = valid_elevation(v) ? v : -32000.0f;
    }
}

void sanitize_level0(ls200_context *ctx, ls200_dem *dem) {
    const long long n = static_cast<long long>(dem->width) * dem->height;
    const int blocks = static_cast<int>(std::min<long long>((n + 255) / 256,
                                                            ctx->props.multiProcessorCount * 8));
    sanitize_kernel<<<blocks, 256, 0, ctx->stream>>>(dem->level0, n, dem->cells);
    LS_CUDA(cudaGetLastError());
}

struct BoundLevels {
    int4 level[kMaxLevels];  // (cell offset, width, height, -), as the march's tables
    int count;
};

// bounds[i] = four_cell_bound of cell i, through the march's own function so
// that the stored value is the one the march would compute.  Grid-stride over
// every cell of every level.
__global__ void cell_bounds_kernel(const float *__restrict__ cells, float *__restrict__ bounds,
                                   const __grid_constant__ BoundLevels T, long long total) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        for (int l = 0; l < T.count; ++l) {
            const int4 L = T.level[l];
            const long long local = i - L.x;
            if (local < 0 || local >= static_cast<long long>(L.y) * L.z) continue;
            const int cy = static_cast<int>(local / L.y);
            const int cx = static_cast<int>(local - static_cast<long long>(cy) * L.y);
            bounds[i] = four_cell_bound(cells, L, cx, cy);
            break;
        }
    }
}

void build_cell_bounds(ls200_context *ctx, ls200_dem *dem) {
    BoundLevels T{};
    const int cells0 = dem->width * dem->height;
    T.count = dem->level_count;
    for (int l = 0; l < dem->level_count; ++l)
        T.level[l] = make_int4(l == 0 ? 0 : cells0 + dem->levels[l].offset,
                               dem->levels[l].width, dem->levels[l].height, 0);
    const long long total = static_cast<long long>(cells0) + dem->mip_count;
    const int blocks = static_cast<int>(std::min<long long>(
        (total + 255) / 256, static_cast<long long>(ctx->props.multiProcessorCount) * 8));
    cell_bounds_kernel<<<blocks, 256, 0, ctx->stream>>>(dem->cells, dem->bounds, T, total);
    LS_CUDA(cudaGetLastError());
}

void build_pyramid_device(ls200_context *ctx, ls200_dem *dem) {
    const float *source = dem->level0;
    int sw = dem->width, sh = dem->height;
    for (int level = 1; level < dem->level_count; ++level) {
        const PyramidLevel &L = dem->levels[level];
        float *destination = dem->mips + L.offset;
        dim3 block(32, 8);
        dim3 grid((L.width + block.x - 1) / block.x, (L.height + block.y - 1) / block.y);
        pyramid_downsample<<<grid, block, 0, ctx->stream>>>(source, sw, sh, destination,
                                                            L.width, L.height);
        LS_CUDA(cudaGetLastError());
        source = destination;
        sw = L.width;
        sh = L.height;
    }
}

}  // namespace ls200
