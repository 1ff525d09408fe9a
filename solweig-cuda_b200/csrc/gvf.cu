// solweig_gvf: the 17 ground-view-factor planes for given shadow / wallsun /
// Tg fields (the reference's gvf(), src/model.py:569-622).
#include "gvf.cuh"

namespace solweig {

constexpr int kGvfBX = 32, kGvfBY = 8;

__global__ void __launch_bounds__(256) gvf_quad_kernel(
    const float* __restrict__ shadow, const double* __restrict__ wallsun,
    const float* __restrict__ tg, const double* __restrict__ walls, const uint8_t* __restrict__ flags,
    const float* __restrict__ emis, const float* __restrict__ alb, long long n, double ta,
    double twater, int has_water, float4* __restrict__ quad, float* __restrict__ lup_first) {
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const uint8_t fl = flags[p];
    const double ground = (fl & 1) ? 1.0 : 0.0;
    const bool sunwall = (wallsun[p] / walls[p] * ground) == 1.0;
    const double sh = shadow[p];
    const double e = emis[p];
    double t = tg[p];
    const double amb = kSBC * e * pow4(ta + 273.15);
    lup_first[p] = (float)(kSBC * e * pow4(t * sh + ta + 273.15) - amb);
    if (has_water && (fl & 4)) t = twater - ta;
    quad[p] = make_float4((float)sh, (float)(kSBC * e * pow4(t * sh + ta + 273.15) - amb), alb[p],
                          __int_as_float(((fl & 1) ? kQuadGround : 0) | (sunwall ? kQuadSunwall : 0)));
}

__global__ void __launch_bounds__(kGvfBX* kGvfBY) gvf_planes_kernel(
    const float4* __restrict__ quad, const float* __restrict__ lup_first,
    const uint32_t* __restrict__ face, const float* __restrict__ emis, int rows, int cols,
    const int2* __restrict__ gofs, GvfScalars gs, int has_water, double ta, float* __restrict__ planes) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    int2* offs = reinterpret_cast<int2*>(smem_raw);
    float4* tile = reinterpret_cast<float4*>(smem_raw + sizeof(int2) * SOLWEIG_GVF_DIRECTIONS * SOLWEIG_GVF_MAX_STEPS);
    const int H = gs.second - 1;
    const int pitch = kGvfBX + 2 * H;
    const int row0 = blockIdx.y * kGvfBY - H, col0 = blockIdx.x * kGvfBX - H;
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    for (int i = tid; i < SOLWEIG_GVF_DIRECTIONS * gs.second; i += blockDim.x * blockDim.y) offs[i] = gofs[i];
    load_quad_tile(tile, pitch, kGvfBY + 2 * H, quad, rows, cols, row0, col0);
    __syncthreads();
    const int c = blockIdx.x * kGvfBX + threadIdx.x;
    const int r = blockIdx.y * kGvfBY + threadIdx.y;
    if (r >= rows || c >= cols) return;
    const long long n = (long long)rows * cols;
    const long long p = (long long)r * cols + c;
    const float4 own = tile[(threadIdx.y + H) * pitch + threadIdx.x + H];
    auto sample = [&](int rr, int cc) -> float4 { return tile[(rr - row0) * pitch + (cc - col0)]; };
    auto lfirst = [&](int rr, int cc) -> float { return __ldg(&lup_first[(long long)rr * cols + cc]); };
    const GvfSums g = gvf_walk(sample, lfirst, has_water != 0, r, c, rows, cols, offs, face[p], own, gs);
    const double amb = kSBC * (double)emis[p] * pow4(ta + 273.15);
    for (int d = 0; d < 5; ++d) {
        const float div = d == 0 ? 18.f : 9.f;
        planes[(3 * d) * n + p] = (float)((double)(g.lup[d] / div) + amb);
        planes[(3 * d + 1) * n + p] = g.alb[d] / div;
        planes[(3 * d + 2) * n + p] = g.nosh[d] / div;
    }
    planes[15 * n + p] = g.gvf_sum;
    planes[16 * n + p] = (__float_as_int(own.w) & kQuadGround) ? g.gvf_sum / 18.f : 1.f;
}

}  // namespace solweig

using namespace solweig;

extern "C" int solweig_gvf(const SolweigScene* scene, const float* shadow, const double* wallsun,
                           const float* tg, double tgwall, double ta, double ewall, double albedo_b,
                           double twater, const int32_t* gvf_dxdy, int first_steps,
                           int second_steps, float* scratch, float* planes, void* stream) {
    SOLWEIG_CHECK_ARG(scene && shadow && wallsun && tg && gvf_dxdy && scratch && planes,
                      "solweig_gvf: null pointer");
    const SolweigScene& S = *scene;
    SOLWEIG_CHECK_ARG(S.walls && S.flags && S.emis && S.alb && S.gvf_face,
                      "solweig_gvf: scene is missing walls/flags/emis/alb/gvf_face");
    SOLWEIG_CHECK_ARG(second_steps >= 1 && second_steps <= SOLWEIG_GVF_MAX_STEPS && first_steps >= 1 &&
                          first_steps <= second_steps,
                      "solweig_gvf: steps first=%d second=%d", first_steps, second_steps);
    const long long n = (long long)S.rows * S.cols;
    const int H = second_steps - 1;
    const size_t smem = sizeof(int2) * SOLWEIG_GVF_DIRECTIONS * SOLWEIG_GVF_MAX_STEPS +
                        sizeof(float4) * (size_t)(kGvfBX + 2 * H) * (kGvfBY + 2 * H);
    SOLWEIG_CHECK_ARG(smem <= 227 * 1024, "solweig_gvf: halo %d too large", H);
    cudaStream_t st = as_stream(stream);
    float4* quad = reinterpret_cast<float4*>(scratch);
    float* lup_first = scratch + 4 * n;
    gvf_quad_kernel<<<blocks_for(n, 256), 256, 0, st>>>(shadow, wallsun, tg, S.walls, S.flags, S.emis,
                                                        S.alb, n, ta, twater, S.has_water, quad,
                                                        lup_first);
    SOLWEIG_CHECK_LAUNCH("gvf_quad_kernel");
    GvfScalars gs;
    gs.lwall = (float)(kSBC * ewall * pow4(tgwall + ta + 273.15) - kSBC * ewall * pow4(ta + 273.15));
    gs.albedo_b = (float)albedo_b;
    gs.first = first_steps;
    gs.second = second_steps;
    dim3 block(kGvfBX, kGvfBY), grid(blocks_for(S.cols, kGvfBX), blocks_for(S.rows, kGvfBY));
    cudaFuncSetAttribute(gvf_planes_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    gvf_planes_kernel<<<grid, block, smem, st>>>(quad, lup_first, S.gvf_face, S.emis, S.rows, S.cols,
                                                 reinterpret_cast<const int2*>(gvf_dxdy), gs,
                                                 S.has_water, ta, planes);
    SOLWEIG_CHECK_LAUNCH("gvf_planes_kernel");
    return SOLWEIG_OK;
}
