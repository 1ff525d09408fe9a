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

// One thread per pixel; non-wall pixels write 0.  Template offset lists are
// small (<= 9 entries per angle for 1 m pixels) and read through L1.
__global__ void __launch_bounds__(256) wall_aspect_kernel(
    const double* __restrict__ dsm, const double* __restrict__ walls, double* __restrict__ aspect,
    int rows, int cols, int radius, const int32_t* __restrict__ line_off,
    const int32_t* __restrict__ line_start, const int32_t* __restrict__ s1_off,
    const int32_t* __restrict__ s1_start, const int32_t* __restrict__ s2_off,
    const int32_t* __restrict__ s2_start) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const int r = blockIdx.y;
    if (c >= cols) return;
    const long long p = (long long)r * cols + c;
    double out = 0.0;
    if (walls[p] > 0.0 && r >= radius && r < rows - radius - 2 && c >= radius &&
        c < cols - radius - 2) {
        int best = 0, best_angle = -1;
        for (int angle = 0; angle < 180; ++angle) {
            int score = 0;
            for (int j = line_start[angle]; j < line_start[angle + 1]; ++j) {
                const int rr = r + line_off[2 * j], cc = c + line_off[2 * j + 1];
                score += walls[(long long)rr * cols + cc] > 0.0 ? 1 : 0;
            }
            if (score > best) {
                best = score;
                best_angle = angle;
            }
        }
        if (best_angle >= 0) {
            double first = 0.0, second = 0.0;
            for (int j = s1_start[best_angle]; j < s1_start[best_angle + 1]; ++j)
                first += dsm[(long long)(r + s1_off[2 * j]) * cols + (c + s1_off[2 * j + 1])];
            for (int j = s2_start[best_angle]; j < s2_start[best_angle + 1]; ++j)
                second += dsm[(long long)(r + s2_off[2 * j]) * cols + (c + s2_off[2 * j + 1])];
            double dir = 270.0 - best_angle;
            if (first > second) dir -= 180.0;
            if (dir < 0.0) dir += 360.0;
            out = dir;
        }
    }
    aspect[p] = out;
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
