// Walls from the DSM: wall heights and the template-based wall aspect.
//
// Heights follow src/kernels/geometry.cu:15-34 (4-neighbour maximum minus the
// cell, kept where >= threshold; border cells zero except the row-0 quirk at
// columns rows <= col < cols-1).  The aspect search follows src/walls.py:83-121
// with geometry.cu:36-63: for every wall pixel the 180 rotated line templates
// are scored by how many wall pixels they cover (first maximum wins), then the
// two side templates of the winning angle decide which way the wall faces.
#include "common.cuh"

namespace solweig {

__global__ void __launch_bounds__(256) wall_heights_kernel(const double* __restrict__ dsm,
                                                           double* __restrict__ walls, int rows,
                                                           int cols, double threshold) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const int r = blockIdx.y;
    if (c >= cols) return;
    const long long p = (long long)r * cols + c;
    double h = 0.0;
    if (r > 0 && r < rows - 1 && c > 0 && c < cols - 1) {
        const double nb = fmax(fmax(dsm[p - cols], dsm[p + cols]), fmax(dsm[p - 1], dsm[p + 1]));
        const double d = nb - dsm[p];
        if (d >= threshold) h = d;
    } else if (r == 0 && rows > 1 && c >= rows && c < cols - 1) {
        const double d = -dsm[p];
        if (d >= threshold) h = d;
    }
    walls[p] = h;
}

// A block covers 256 pixels of one row, one lane per pixel; non-wall pixels
// write 0.  Wall pixels are few (a row segment of 32 holds a couple), so the
// warp takes its wall pixels one after another and spreads the 180 template
// angles over its lanes (angle = lane + 32 i); the best angle is the first
// one with the highest score (scores compared strictly, as the per-pixel loop
// does), found by a warp maximum of the scores and a minimum of the angles
// that reach it.  The side sums of the chosen angle are added by the pixel's
// own lane in the template's order.  Template offset lists are small (<= 9
// entries per angle for 1 m pixels) and read through L1.
__global__ void __launch_bounds__(256) wall_aspect_kernel(
    const double* __restrict__ dsm, const double* __restrict__ walls, double* __restrict__ aspect,
    int rows, int cols, int radius, const int32_t* __restrict__ line_off,
    const int32_t* __restrict__ line_start, const int32_t* __restrict__ s1_off,
    const int32_t* __restrict__ s1_start, const int32_t* __restrict__ s2_off,
    const int32_t* __restrict__ s2_start) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const int r = blockIdx.y;
    const int lane = threadIdx.x & 31;
    const bool in = c < cols;
    const long long p = (long long)r * cols + (in ? c : 0);
    const bool cand = in && walls[p] > 0.0 && r >= radius && r < rows - radius - 2 && c >= radius &&
                      c < cols - radius - 2;
    double out = 0.0;
    for (uint32_t m = __ballot_sync(0xffffffffu, cand); m; m &= m - 1) {
        const int src = __ffs(m) - 1;
        const int pc = __shfl_sync(0xffffffffu, c, src);
        int best = 0, best_angle = -1;
        for (int angle = lane; angle < 180; angle += 32) {
            int score = 0;
            for (int j = line_start[angle]; j < line_start[angle + 1]; ++j) {
                const int rr = r + line_off[2 * j], cc = pc + line_off[2 * j + 1];
                score += walls[(long long)rr * cols + cc] > 0.0 ? 1 : 0;
            }
            if (score > best) {
                best = score;
                best_angle = angle;
            }
        }
        const int top = __reduce_max_sync(0xffffffffu, best);
        const int first = __reduce_min_sync(0xffffffffu, (best == top && best_angle >= 0) ? best_angle : 1 << 30);
        if (lane == src && top > 0) {
            double s1 = 0.0, s2 = 0.0;
            for (int j = s1_start[first]; j < s1_start[first + 1]; ++j)
                s1 += dsm[(long long)(r + s1_off[2 * j]) * cols + (pc + s1_off[2 * j + 1])];
            for (int j = s2_start[first]; j < s2_start[first + 1]; ++j)
                s2 += dsm[(long long)(r + s2_off[2 * j]) * cols + (pc + s2_off[2 * j + 1])];
            double dir = 270.0 - first;
            if (s1 > s2) dir -= 180.0;
            if (dir < 0.0) dir += 360.0;
            out = dir;
        }
    }
    if (in) aspect[p] = out;
}

}  // namespace solweig

using namespace solweig;

extern "C" int solweig_wall_heights(const double* dsm, double* walls, int rows, int cols,
                                    double threshold, void* stream) {
    SOLWEIG_CHECK_ARG(dsm && walls, "solweig_wall_heights: null pointer");
    SOLWEIG_CHECK_ARG(rows > 0 && cols > 0 && rows < 65536, "solweig_wall_heights: bad shape %dx%d",
                      rows, cols);
    dim3 grid(blocks_for(cols, 256), rows);
    wall_heights_kernel<<<grid, 256, 0, as_stream(stream)>>>(dsm, walls, rows, cols, threshold);
    SOLWEIG_CHECK_LAUNCH("wall_heights_kernel");
    return SOLWEIG_OK;
}

extern "C" int solweig_wall_aspect(const double* dsm, const double* walls, double* aspect, int rows,
                                   int cols, int radius, const int32_t* line_off,
                                   const int32_t* line_start, const int32_t* side1_off,
                                   const int32_t* side1_start, const int32_t* side2_off,
                                   const int32_t* side2_start, void* stream) {
    SOLWEIG_CHECK_ARG(dsm && walls && aspect && line_off && line_start && side1_off && side1_start &&
                          side2_off && side2_start,
                      "solweig_wall_aspect: null pointer");
    SOLWEIG_CHECK_ARG(rows > 0 && cols > 0 && rows < 65536 && radius >= 1,
                      "solweig_wall_aspect: bad shape %dx%d radius %d", rows, cols, radius);
    dim3 grid(blocks_for(cols, 256), rows);
    wall_aspect_kernel<<<grid, 256, 0, as_stream(stream)>>>(dsm, walls, aspect, rows, cols, radius,
                                                            line_off, line_start, side1_off,
                                                            side1_start, side2_off, side2_start);
    SOLWEIG_CHECK_LAUNCH("wall_aspect_kernel");
    return SOLWEIG_OK;
}
