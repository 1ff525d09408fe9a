// Walls from building footprints: the geometry wall method of
// src/walls.py:270-332 (calculate_geometry_walls).  Every polygon edge is a
// wall segment with its building's height and its outward aspect; the
// reference burns the segments into the raster with rasterio.features.
// rasterize (all_touched, later shapes replace earlier ones) once for the
// mask, once for the heights and once for the aspects, then prefers the GHSL
// height where it reaches the minimum wall height.
//
// Here one pass burns them all: a thread walks one segment through the cells
// it touches and raises each cell's owner to its segment index (atomicMax),
// so the last segment touching a cell owns it, as with "replace"; a second
// pass per pixel turns owners into the mask, height and aspect planes.
//
// Touching is defined on pixel coordinates (u, v) = the inverse geotransform
// of (x, y): cell (col, row) is the half-open square [col, col + 1) x
// [row, row + 1), and a segment touches every cell that holds one of its
// points.  The walk is a grid traversal whose crossing order is decided by
// comparing cross products (|X - u0| |dv| against |Y - v0| |du|), so it is
// exact whenever those products are (coordinates on a binary grid): a
// crossing in the increasing direction happens at the boundary point itself,
// one in the decreasing direction just after it, which fixes the order at
// corners.
#include "common.cuh"

namespace solweig {

__global__ void __launch_bounds__(256) segment_burn_kernel(const double4* __restrict__ seg, int nseg, int rows,
                                                           int cols, int* __restrict__ owner) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nseg) return;
    const double4 g = seg[s];
    const double u0 = g.x, v0 = g.y, u1 = g.z, v1 = g.w;
    if (!(isfinite(u0) && isfinite(v0) && isfinite(u1) && isfinite(v1))) return;
    // Segments whose box misses the raster touch none of its cells; the walk
    // below only visits cells between the two end cells.
    if (fmax(u0, u1) < 0.0 || fmin(u0, u1) >= (double)cols || fmax(v0, v1) < 0.0 ||
        fmin(v0, v1) >= (double)rows)
        return;
    const double du = u1 - u0, dv = v1 - v0;
    const int sx = (du > 0.0) - (du < 0.0), sy = (dv > 0.0) - (dv < 0.0);
    const double adu = fabs(du), adv = fabs(dv);
    long long ci = (long long)floor(u0), cj = (long long)floor(v0);
    const long long ei = (long long)floor(u1), ej = (long long)floor(v1);
    const long long steps = llabs(ei - ci) + llabs(ej - cj);
    for (long long k = 0; k <= steps; ++k) {
        if (ci >= 0 && ci < cols && cj >= 0 && cj < rows) atomicMax(&owner[cj * (long long)cols + ci], s);
        if (ci == ei && cj == ej) break;
        bool step_x, step_y;
        if (sx == 0) {
            step_x = false;
            step_y = true;
        } else if (sy == 0) {
            step_x = true;
            step_y = false;
        } else {
            const double X = sx > 0 ? (double)(ci + 1) : (double)ci;
            const double Y = sy > 0 ? (double)(cj + 1) : (double)cj;
            const double tx = fabs(X - u0) * adv;  // crossing time of the column boundary x |du||dv|
            const double ty = fabs(Y - v0) * adu;
            if (tx < ty) {
                step_x = true;
                step_y = false;
            } else if (ty < tx) {
                step_x = false;
                step_y = true;
            } else if (sx == sy) {  // both crossings at (or both just after) the corner
                step_x = step_y = true;
            } else {  // the increasing crossing happens first
                step_x = sx > 0;
                step_y = !step_x;
            }
        }
        if (step_x) ci += sx;
        if (step_y) cj += sy;
    }
}

// numpy's float32 remainder by 360 (sign of the divisor).
__device__ __forceinline__ float remainder360(float a) {
    float r = fmodf(a, 360.0f);
    if (r != 0.0f && r < 0.0f) r += 360.0f;
    return r == 0.0f ? 0.0f : r;
}

__global__ void __launch_bounds__(256) geometry_walls_kernel(const int* __restrict__ owner,
                                                             const double* __restrict__ height,
                                                             const double* __restrict__ aspect_deg,
                                                             const float* __restrict__ ghsl, long long n,
                                                             float minimum, float* __restrict__ walls,
                                                             float* __restrict__ aspect) {
    const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (p >= n) return;
    const int o = owner[p];
    if (o < 0) {
        walls[p] = 0.0f;
        aspect[p] = 0.0f;
        return;
    }
    float gh = ghsl ? ghsl[p] : 0.0f;
    if (!isfinite(gh)) gh = 0.0f;  // nan_to_num
    walls[p] = gh >= minimum ? gh : (float)height[o];
    aspect[p] = remainder360((float)aspect_deg[o]);
}

}  // namespace solweig

using namespace solweig;

extern "C" int solweig_wall_segments_burn(const double* segments, int64_t nseg, int rows, int cols,
                                          int32_t* owner, void* stream) {
    SOLWEIG_CHECK_ARG(owner && (segments || nseg == 0), "solweig_wall_segments_burn: null pointer");
    SOLWEIG_CHECK_ARG(rows > 0 && cols > 0 && nseg >= 0 && nseg < (1ll << 31),
                      "solweig_wall_segments_burn: bad sizes %dx%d, %lld segments", rows, cols, (long long)nseg);
    SOLWEIG_CHECK_ARG(((uintptr_t)segments & 15) == 0, "solweig_wall_segments_burn: segments not 16-byte aligned");
    cudaStream_t st = as_stream(stream);
    cudaMemsetAsync(owner, 0xff, sizeof(int32_t) * (size_t)rows * cols, st);
    SOLWEIG_CHECK_LAUNCH("solweig_wall_segments_burn: clear");
    if (nseg == 0) return SOLWEIG_OK;
    segment_burn_kernel<<<blocks_for(nseg, 256), 256, 0, st>>>(reinterpret_cast<const double4*>(segments),
                                                                (int)nseg, rows, cols, owner);
    SOLWEIG_CHECK_LAUNCH("segment_burn_kernel");
    return SOLWEIG_OK;
}

extern "C" int solweig_geometry_walls(const int32_t* owner, const double* seg_height, const double* seg_aspect,
                                      const float* ghsl, int64_t pixels, double minimum, float* walls,
                                      float* aspect, void* stream) {
    SOLWEIG_CHECK_ARG(owner && walls && aspect && pixels >= 0, "solweig_geometry_walls: bad arguments");
    if (pixels == 0) return SOLWEIG_OK;
    geometry_walls_kernel<<<blocks_for(pixels, 256), 256, 0, as_stream(stream)>>>(
        owner, seg_height, seg_aspect, ghsl, pixels, (float)minimum, walls, aspect);
    SOLWEIG_CHECK_LAUNCH("geometry_walls_kernel");
    return SOLWEIG_OK;
}
