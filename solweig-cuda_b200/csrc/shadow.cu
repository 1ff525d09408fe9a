// solweig_shadow: the eight shadow planes of one sun position (cast_shadow).
#include "shadow.cuh"

namespace solweig {

// Block = 32 columns x 8 rows: a warp reads one contiguous 32-column run per
// ray step, and the 8 warps of a block walk parallel rays one row apart, so
// consecutive steps of neighbouring warps hit the same cache lines.
constexpr int kShadowBX = 32, kShadowBY = 8;

__global__ void __launch_bounds__(kShadowBX* kShadowBY) shadow_planes_kernel(
    const double* __restrict__ dsm, const double* __restrict__ top, const double* __restrict__ bot,
    const double* __restrict__ walls, const double* __restrict__ aspect,
    const uint8_t* __restrict__ flags, int rows, int cols, const int2* __restrict__ ray,
    const double* __restrict__ dz, int steps, double hmax, double low, double high, int middle,
    int vegetation, double* __restrict__ out) {
    const int c = blockIdx.x * kShadowBX + threadIdx.x;
    const int r = blockIdx.y * kShadowBY + threadIdx.y;
    if (r >= rows || c >= cols) return;
    const long long n = (long long)rows * cols;
    const long long p = (long long)r * cols + c;
    const double a = dsm[p];
    const double wall = walls[p];
    const bool bush = vegetation && (flags[p] & 2);
    const double top_p = vegetation ? top[p] : 0.0;
    ShadowResult s = shadow_walk(dsm, top, bot, rows, cols, r, c, a, top_p, bush, wall, ray, dz,
                                 steps, hmax, vegetation != 0);
    const double wallbol = wall > 0.0 ? 1.0 : 0.0;
    const double facesh = self_shadow_face(aspect[p], wallbol, low, high, middle);
    const double volume = s.f - a;
    double wallsun = wall - volume;
    if (wallsun < 0.0) wallsun = 0.0;
    if (facesh == 1.0) wallsun = 0.0;
    const double wallsh = wall - wallsun;
    double wallshve = 0.0;
    if (vegetation) {
        const double vegf = s.veg ? 1.0 : 0.0;
        wallshve = (s.topmax - a) * vegf * wallbol - wallsh;
        if (wallshve < 0.0) wallshve = 0.0;
        if (wallshve > wall) wallshve = wall;
        wallsun = wallsun - wallshve;
        if (wallsun < 0.0) {
            wallshve = 0.0;
            wallsun = 0.0;
        }
    }
    out[p] = 1.0 - (s.veg ? 1.0 : 0.0);
    out[n + p] = vegetation ? 1.0 - (s.shadowed ? 1.0 : 0.0) : 1.0 - (volume != 0.0 ? 1.0 : 0.0);
    out[2 * n + p] = 1.0 - ((s.ever ? 1.0 : 0.0) - (s.veg ? 1.0 : 0.0));
    out[3 * n + p] = wallsh;
    out[4 * n + p] = wallsun;
    out[5 * n + p] = wallshve;
    out[6 * n + p] = facesh;
    out[7 * n + p] = (facesh + wallbol == 1.0 && wall > 0.0) ? 1.0 : 0.0;
}

}  // namespace solweig

using namespace solweig;

extern "C" int solweig_shadow(const SolweigScene* scene, const int32_t* ray_dxdy,
                              const double* ray_dz, int steps, double low, double high, int middle,
                              int vegetation, double* out, void* stream) {
    SOLWEIG_CHECK_ARG(scene && ray_dxdy && ray_dz && out, "solweig_shadow: null pointer");
    SOLWEIG_CHECK_ARG(scene->dsm && scene->walls && scene->aspect && scene->flags,
                      "solweig_shadow: scene is missing dsm/walls/aspect/flags");
    SOLWEIG_CHECK_ARG(!vegetation || (scene->vegdem && scene->vegdem2),
                      "solweig_shadow: vegetation needs vegdem and vegdem2");
    SOLWEIG_CHECK_ARG(scene->rows > 0 && scene->cols > 0 && steps >= 0,
                      "solweig_shadow: bad shape or step count");
    dim3 block(kShadowBX, kShadowBY);
    dim3 grid(blocks_for(scene->cols, kShadowBX), blocks_for(scene->rows, kShadowBY));
    shadow_planes_kernel<<<grid, block, 0, as_stream(stream)>>>(
        scene->dsm, scene->vegdem, scene->vegdem2, scene->walls, scene->aspect, scene->flags,
        scene->rows, scene->cols, reinterpret_cast<const int2*>(ray_dxdy), ray_dz, steps,
        scene->hmax, low, high, middle, vegetation, out);
    SOLWEIG_CHECK_LAUNCH("shadow_planes_kernel");
    return SOLWEIG_OK;
}
