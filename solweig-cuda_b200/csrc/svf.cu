// Sky view factor: per-patch visibility rays, bit-packed, and the annulus sums.
//
// Visibility (src/kernels/geometry.cu:77-119, src/svf.py:81-106): for every
// pixel and sky patch the shadow sweep toward the patch centre decides whether
// a building blocks the patch (S = 0) and whether vegetation was seen in front
// of the first building hit (V = 1).  The reference stores three float32
// cubes [rows, cols, 153] (7.3 GB at 2000^2); here each (pixel, patch) keeps
// 2 bits, 40 bytes per pixel, in the layout described in solweig_b200.h.
//
// Reduce (geometry.cu:121-159): annulus-weighted sums over bands and the four
// half-sky sectors become per-band popcounts of the packed words, summed in
// the reference's band order so the float64 planes agree to the last bit.
#include "ceiling.cuh"
#include "shadow.cuh"

namespace solweig {

constexpr int kSvfWarps = 8;        // warps per block
constexpr int kSvfPatchGroup = 32;  // patches per packed word

struct SvfRayParams {
    int rows, cols, patches, capacity;
    double hmax;
};

// grid.x: chunks of 32 consecutive pixels; grid.y: patch word (32 patches)
// from word0 on.  geo32: the packed float4 geometry (exact float32 values) or
// null.  With `ceiling` and `exits` (one launch per word, grid.y = 1): the
// word's ray-ceiling planes [32][pixels] and first-outside steps [32][rows +
// cols]; the walk then stops on the ceilings and, with geo32, needs no
// bounds checks.
// WALK: 0 float64 rasters, 1 packed geometry, 2 packed geometry without
// bounds checks (`exits` given; used when the step records do not fit, else
// svf_visibility_warp_kernel).
// 32 registers (8 blocks per SM): the walks are latency-bound and full
// occupancy outweighs the few spills (SVF 5.7 ms faster at 2000^2 than at
// 40 registers).
template <int WALK>
__global__ void __launch_bounds__(32 * kSvfWarps, 8) svf_visibility_kernel(
    const double* __restrict__ dsm, const double* __restrict__ top, const double* __restrict__ bot,
    const float4* __restrict__ geo32, const uint8_t* __restrict__ flags, SvfRayParams prm,
    const int2* __restrict__ ray, const double* __restrict__ dz, const int32_t* __restrict__ lengths,
    uint32_t* __restrict__ masks, int word0, const float2* __restrict__ ceiling, const int* __restrict__ exits) {
    __shared__ uint8_t state[kSvfPatchGroup][32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const long long pixels = (long long)prm.rows * prm.cols;
    // the block's 32 pixels: an 8 x 4 (columns x rows) tile, whose walks are
    // more alike than those of 32 pixels in a row
    const int tiles_x = (prm.cols + 7) / 8;
    const int rr = (blockIdx.x / tiles_x) * 4 + (lane >> 3), cc = (blockIdx.x % tiles_x) * 8 + (lane & 7);
    const int word = word0 + blockIdx.y;
    const bool valid = rr < prm.rows && cc < prm.cols;
    const int r = valid ? rr : 0, c = valid ? cc : 0;
    const long long p = (long long)r * prm.cols + c;
    const double a = valid ? dsm[p] : 0.0;
    const double top_p = valid ? top[p] : 0.0;
    const bool bush = valid && (flags[p] & 2);
    for (int j = warp; j < kSvfPatchGroup; j += kSvfWarps) {
        const int patch = word * kSvfPatchGroup + j;
        uint8_t st = 0;
        if (valid && patch < prm.patches) {
            const long long base = (long long)patch * prm.capacity;
            const int K = lengths[patch];
            const float2* ceil_j = ceiling ? ceiling + (long long)j * pixels : nullptr;
            ShadowResult s;
            if (WALK == 2) {
                const int* e = exits + (long long)j * (prm.rows + prm.cols);
                const int kend = min(K, min(__ldg(&e[r]), __ldg(&e[prm.rows + c])));
                s = shadow_walk_packed<false>(geo32, prm.cols, p, a, top_p, bush, 0.0, ray + base, dz + base,
                                              nullptr, K, kend, prm.hmax, ceil_j);
            } else if (WALK == 1) {
                s = shadow_walk_geo(GeoF32x4{geo32}, prm.rows, prm.cols, r, c, a, top_p, bush, 0.0, ray + base,
                                    dz + base, K, prm.hmax, true, ceil_j);
            } else {
                s = shadow_walk_geo(GeoF64{dsm, top, bot}, prm.rows, prm.cols, r, c, a, top_p, bush, 0.0,
                                    ray + base, dz + base, K, prm.hmax, true, ceil_j);
            }
            st = (s.shadowed ? 0 : 1) | (s.ever ? 2 : 0);
        }
        state[j][lane] = st;
    }
    __syncthreads();
    if (warp < 2 && valid) {
        uint32_t bits = 0;
#pragma unroll
        for (int j = 0; j < kSvfPatchGroup; ++j) bits |= (uint32_t)((state[j][lane] >> warp) & 1u) << j;
        masks[((long long)warp * SOLWEIG_MASK_WORDS + word) * pixels + p] = bits;
    }
}

// The step-record form (WALK 3) with one warp per 8 x 4 pixel tile walking
// all patches of the word in turn (grid.x: tiles / 8, one word per launch):
// the warps of a block carry similar work -- each walks all 32 patches of
// its own pixels, so the uneven lengths of single walks (window skips,
// ceiling exits) even out -- and each pixel's two bits are assembled in
// registers, so no warp waits at a barrier.  Same walks, same bits.
__global__ void __launch_bounds__(32 * kSvfWarps, 8) svf_visibility_warp_kernel(
    const float4* __restrict__ geo32, const uint8_t* __restrict__ flags, SvfRayParams prm,
    const int32_t* __restrict__ lengths, uint32_t* __restrict__ masks, int word, const float2* __restrict__ ceiling,
    const int* __restrict__ exits, const longlong2* __restrict__ rec, int kmax) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const long long pixels = (long long)prm.rows * prm.cols;
    const int tiles_x = (prm.cols + 7) / 8;
    const long long ntiles = (long long)tiles_x * ((prm.rows + 3) / 4);
    const long long tile = (long long)blockIdx.x * kSvfWarps + warp;
    if (tile >= ntiles) return;  // the whole warp
    const int rr = (int)(tile / tiles_x) * 4 + (lane >> 3), cc = (int)(tile % tiles_x) * 8 + (lane & 7);
    if (rr >= prm.rows || cc >= prm.cols) return;
    const long long p = (long long)rr * prm.cols + cc;
    const float4 g = __ldg(&geo32[p]);  // the packed geometry holds the exact heights
    const double a = g.x, top_p = g.y;
    const bool bush = flags[p] & 2;
    uint32_t sbits = 0u, vbits = 0u;
    for (int j = 0; j < kSvfPatchGroup; ++j) {
        const int patch = word * kSvfPatchGroup + j;
        if (patch >= prm.patches) break;
        const int K = lengths[patch];
        const int* e = exits + (long long)j * (prm.rows + prm.cols);
        const int kend = min(K, min(__ldg(&e[rr]), __ldg(&e[prm.rows + cc])));
        const ShadowResult s = shadow_walk_packed<true>(geo32, prm.cols, p, a, top_p, bush, 0.0, nullptr, nullptr,
                                                        rec + (long long)j * kmax, K, kend, prm.hmax,
                                                        ceiling + (long long)j * pixels);
        sbits |= (s.shadowed ? 0u : 1u) << j;
        vbits |= (s.ever ? 1u : 0u) << j;
    }
    masks[(long long)word * pixels + p] = sbits;
    masks[((long long)SOLWEIG_MASK_WORDS + word) * pixels + p] = vbits;
}

struct SvfReduceParams {
    long long pixels;
    int nbands;
    double trans;
    uint32_t band_mask[SOLWEIG_MAX_BANDS][SOLWEIG_MASK_WORDS];
    uint32_t sector_mask[4][SOLWEIG_MASK_WORDS];
    double wf[SOLWEIG_MAX_BANDS], wa[SOLWEIG_MAX_BANDS];
    double w_cos[SOLWEIG_MAX_BANDS], w_sin[SOLWEIG_MAX_BANDS];  // omega*cos, omega*sin per band
};

__global__ void __launch_bounds__(256) svf_reduce_kernel(const uint32_t* __restrict__ masks,
                                                         const double* __restrict__ bot,
                                                         SvfReduceParams prm,
                                                         double* __restrict__ planes,
                                                         float* __restrict__ veg_sums,
                                                         uint8_t* __restrict__ sky_counts) {
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= prm.pixels) return;
    const long long n = prm.pixels;
    uint32_t S[SOLWEIG_MASK_WORDS], V[SOLWEIG_MASK_WORDS];
#pragma unroll
    for (int w = 0; w < SOLWEIG_MASK_WORDS; ++w) {
        S[w] = masks[(long long)w * n + p];
        V[w] = masks[(long long)(SOLWEIG_MASK_WORDS + w) * n + p];
    }
    double v[15];
#pragma unroll
    for (int i = 0; i < 15; ++i) v[i] = 0.0;
    double vc = 0.0, vs = 0.0, oc = 0.0, os = 0.0;
    for (int b = 0; b < prm.nbands; ++b) {
        int cnt[15];
#pragma unroll
        for (int i = 0; i < 15; ++i) cnt[i] = 0;
        int nveg = 0, nobst = 0, nsky = 0;
#pragma unroll
        for (int w = 0; w < SOLWEIG_MASK_WORDS; ++w) {
            const uint32_t bm = prm.band_mask[b][w];
            const uint32_t sh = S[w] & bm;                // shmat == 1
            const uint32_t vg = ~(S[w] & V[w]) & bm;      // vegmat == 1
            const uint32_t vb = ~(~S[w] & V[w]) & bm;     // vbmat == 1
            cnt[0] += __popc(sh);
            cnt[5] += __popc(vg);
            cnt[10] += __popc(vb);
#pragma unroll
            for (int d = 0; d < 4; ++d) {
                const uint32_t sm = prm.sector_mask[d][w];
                cnt[1 + d] += __popc(sh & sm);
                cnt[6 + d] += __popc(vg & sm);
                cnt[11 + d] += __popc(vb & sm);
            }
            nveg += __popc(V[w] & bm);
            nobst += __popc(~(S[w] & ~V[w]) & bm);
            nsky += __popc(S[w] & ~V[w] & bm);
        }
#pragma unroll
        for (int g = 0; g < 3; ++g) {
            v[g * 5] += prm.wf[b] * cnt[g * 5];
#pragma unroll
            for (int d = 1; d < 5; ++d) v[g * 5 + d] += prm.wa[b] * cnt[g * 5 + d];
        }
        vc += prm.w_cos[b] * nveg;
        vs += prm.w_sin[b] * nveg;
        oc += prm.w_cos[b] * nobst;
        os += prm.w_sin[b] * nobst;
        sky_counts[(long long)b * n + p] = (uint8_t)nsky;
    }
    const double eps = 3.0459e-4;
    v[2] += eps;
    v[3] += eps;
    const double last = bot[p] == 0.0 ? eps : 0.0;
    v[7] += last;
    v[8] += last;
    v[12] += last;
    v[13] += last;
#pragma unroll
    for (int i = 0; i < 15; ++i) {
        if (v[i] > 1.0) v[i] = 1.0;
        planes[(long long)i * n + p] = v[i];
    }
    planes[15 * n + p] = v[0] - (1.0 - v[5]) * (1.0 - prm.trans);
    veg_sums[p] = (float)vc;
    veg_sums[n + p] = (float)vs;
    veg_sums[2 * n + p] = (float)oc;
    veg_sums[3 * n + p] = (float)os;
}

// Packed masks -> the reference's float cubes [pixels][patches].
__global__ void __launch_bounds__(256) svf_unpack_kernel(const uint32_t* __restrict__ masks,
                                                         long long pixels, int patches,
                                                         float* __restrict__ shm,
                                                         float* __restrict__ vegm,
                                                         float* __restrict__ vbm) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= pixels * patches) return;
    const long long p = i / patches;
    const int k = (int)(i % patches);
    const int w = k >> 5, b = k & 31;
    const bool S = (masks[(long long)w * pixels + p] >> b) & 1u;
    const bool V = (masks[(long long)(SOLWEIG_MASK_WORDS + w) * pixels + p] >> b) & 1u;
    if (shm) shm[i] = S ? 1.f : 0.f;
    if (vegm) vegm[i] = (S && V) ? 0.f : 1.f;
    if (vbm) vbm[i] = (!S && V) ? 0.f : 1.f;
}

// Reference float cubes [pixels][patches] -> packed S/V words.
__global__ void __launch_bounds__(256) svf_pack_kernel(const float* __restrict__ shm,
                                                       const float* __restrict__ vegm,
                                                       const float* __restrict__ vbm,
                                                       long long pixels, int patches,
                                                       uint32_t* __restrict__ masks) {
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= pixels) return;
    for (int w = 0; w < SOLWEIG_MASK_WORDS; ++w) {
        uint32_t s = 0, v = 0;
        for (int b = 0; b < 32; ++b) {
            const int k = w * 32 + b;
            if (k >= patches) break;
            const long long i = p * patches + k;
            if (shm[i] == 1.0f) s |= 1u << b;
            if (vegm[i] == 0.0f || vbm[i] == 0.0f) v |= 1u << b;
        }
        masks[(long long)w * pixels + p] = s;
        masks[(long long)(SOLWEIG_MASK_WORDS + w) * pixels + p] = v;
    }
}

__global__ void __launch_bounds__(256) diffsh_kernel(const float* __restrict__ sh,
                                                     const float* __restrict__ veg,
                                                     float* __restrict__ out, long long n,
                                                     float trans) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[i] = __fsub_rn(sh[i], __fmul_rn(__fsub_rn(1.0f, veg[i]), __fsub_rn(1.0f, trans)));
}

}  // namespace solweig

using namespace solweig;

extern "C" int solweig_svf_reduce(const uint32_t* masks, const double* vegdem2, int64_t pixels,
                                  const SolweigSkyLayout* layout, const double* band_weights,
                                  const uint8_t* sectors, double transmissivity, double* planes,
                                  float* veg_sums, uint8_t* sky_band_counts, void* stream) {
    SOLWEIG_CHECK_ARG(masks && vegdem2 && layout && band_weights && sectors && planes && veg_sums &&
                          sky_band_counts && pixels > 0,
                      "solweig_svf_reduce: bad arguments");
    SOLWEIG_CHECK_ARG(layout->nbands > 0 && layout->nbands <= SOLWEIG_MAX_BANDS &&
                          layout->patches > 0 && layout->patches <= SOLWEIG_MASK_WORDS * 32,
                      "solweig_svf_reduce: bad layout");
    const int patches = layout->patches;
    cudaStream_t st = as_stream(stream);
    SvfReduceParams q{};
    q.pixels = pixels;
    q.nbands = layout->nbands;
    q.trans = transmissivity;
    for (int k = 0; k < patches; ++k) {
        const int b = layout->band_of_patch[k];
        SOLWEIG_CHECK_ARG(b >= 0 && b < layout->nbands, "solweig_svf: bad band of patch %d", k);
        q.band_mask[b][k >> 5] |= 1u << (k & 31);
        for (int d = 0; d < 4; ++d)
            if (sectors[k] & (1u << d)) q.sector_mask[d][k >> 5] |= 1u << (k & 31);
    }
    for (int b = 0; b < layout->nbands; ++b) {
        q.wf[b] = band_weights[2 * b];
        q.wa[b] = band_weights[2 * b + 1];
        q.w_cos[b] = (double)layout->band_omega[b] * (double)layout->band_cos[b];
        q.w_sin[b] = (double)layout->band_omega[b] * (double)layout->band_sin[b];
    }
    svf_reduce_kernel<<<blocks_for(pixels, 256), 256, 0, st>>>(masks, vegdem2, q, planes, veg_sums,
                                                               sky_band_counts);
    SOLWEIG_CHECK_LAUNCH("svf_reduce_kernel");
    return SOLWEIG_OK;
}

extern "C" int solweig_svf_pack(const float* shmat, const float* vegmat, const float* vbmat,
                                int64_t pixels, int patches, uint32_t* masks, void* stream) {
    SOLWEIG_CHECK_ARG(shmat && vegmat && vbmat && masks && pixels > 0 && patches > 0 &&
                          patches <= SOLWEIG_MASK_WORDS * 32,
                      "solweig_svf_pack: bad arguments");
    svf_pack_kernel<<<blocks_for(pixels, 256), 256, 0, as_stream(stream)>>>(shmat, vegmat, vbmat,
                                                                           pixels, patches, masks);
    SOLWEIG_CHECK_LAUNCH("svf_pack_kernel");
    return SOLWEIG_OK;
}

// Blocks of the visibility kernel: 8 x 4 pixel tiles.
unsigned svf_tiles(int rows, int cols) { return (unsigned)(((cols + 7) / 8) * ((rows + 3) / 4)); }

// first_outside tables of a group of patches: block j = patch0 + j; with
// rec also the patches' step records (kmax >= every length).
__global__ void __launch_bounds__(1024) patch_ray_exits_kernel(int rows, int cols, const int2* __restrict__ rays,
                                                               const double* __restrict__ dz,
                                                               const int32_t* __restrict__ lengths, int capacity,
                                                               int patch0, int count, int* __restrict__ exits,
                                                               longlong2* __restrict__ rec, int kmax) {
    const int j = blockIdx.x;
    if (j >= count) return;
    const int patch = patch0 + j;
    ray_exits_block(rays + (long long)patch * capacity, lengths[patch], rows, cols,
                    exits + (long long)j * (rows + cols));
    if (rec != nullptr)
        ray_records_block(rays + (long long)patch * capacity, dz + (long long)patch * capacity,
                          min(lengths[patch], kmax), cols, rec + (long long)j * kmax);
}

// Work of solweig_svf_ex2: 4 dilated height planes, the 32 ray-ceiling
// planes (ceiling and window maximum per pixel) of one patch word, its 32 first-outside tables and its step
// records (kmax = max(rows, cols) + 2 per patch, >= every ray's length).
struct SvfWork {
    long long dil, ceil, exits, rec, total;
    int kmax;
};

SvfWork svf_work_layout(int rows, int cols) {
    const long long px = (long long)rows * cols;
    SvfWork w{};
    w.kmax = (rows > cols ? rows : cols) + 2;
    w.dil = 0;
    w.ceil = (4LL * 4 * px + 255) & ~255LL;
    w.exits = (w.ceil + 8LL * kSvfPatchGroup * px + 255) & ~255LL;
    w.rec = (w.exits + 4LL * kSvfPatchGroup * (rows + cols) + 255) & ~255LL;
    w.total = w.rec + 16LL * kSvfPatchGroup * w.kmax;
    return w;
}

extern "C" int64_t solweig_svf_work_bytes(int rows, int cols) {
    if (rows <= 0 || cols <= 0) return 0;
    return svf_work_layout(rows, cols).total;
}

int svf_impl(const double* dsm, const double* vegdem, const double* vegdem2, const void* geo32,
             const uint8_t* flags, int rows, int cols, int patches, int capacity, const int32_t* ray_dxdy,
             const double* ray_dz, const int32_t* lengths, double hmax, const SolweigSkyLayout* layout,
             const double* band_weights, const uint8_t* sectors, double transmissivity, uint32_t* masks,
             double* planes, float* veg_sums, uint8_t* sky_band_counts, void* work, int64_t work_bytes,
             void* stream);

extern "C" int solweig_svf_ex(const double* dsm, const double* vegdem, const double* vegdem2,
                              const void* geo32, const uint8_t* flags, int rows, int cols, int patches,
                              int capacity, const int32_t* ray_dxdy, const double* ray_dz,
                              const int32_t* lengths, double hmax, const SolweigSkyLayout* layout,
                              const double* band_weights, const uint8_t* sectors, double transmissivity,
                              uint32_t* masks, double* planes, float* veg_sums, uint8_t* sky_band_counts,
                              void* stream) {
    return svf_impl(dsm, vegdem, vegdem2, geo32, flags, rows, cols, patches, capacity, ray_dxdy, ray_dz, lengths,
                    hmax, layout, band_weights, sectors, transmissivity, masks, planes, veg_sums, sky_band_counts,
                    nullptr, 0, stream);
}

// solweig_svf_ex with a work buffer of solweig_svf_work_bytes (no counterpart
// in the reference): per patch word, ray ceilings and first-outside tables
// let the visibility walks stop early with identical masks.
extern "C" int solweig_svf_ex2(const double* dsm, const double* vegdem, const double* vegdem2,
                               const void* geo32, const uint8_t* flags, int rows, int cols, int patches,
                               int capacity, const int32_t* ray_dxdy, const double* ray_dz,
                               const int32_t* lengths, double hmax, const SolweigSkyLayout* layout,
                               const double* band_weights, const uint8_t* sectors, double transmissivity,
                               uint32_t* masks, double* planes, float* veg_sums, uint8_t* sky_band_counts,
                               void* work, int64_t work_bytes, void* stream) {
    SOLWEIG_CHECK_ARG(work, "solweig_svf_ex2: null work buffer");
    return svf_impl(dsm, vegdem, vegdem2, geo32, flags, rows, cols, patches, capacity, ray_dxdy, ray_dz, lengths,
                    hmax, layout, band_weights, sectors, transmissivity, masks, planes, veg_sums, sky_band_counts,
                    work, work_bytes, stream);
}

int svf_impl(const double* dsm, const double* vegdem, const double* vegdem2, const void* geo32,
             const uint8_t* flags, int rows, int cols, int patches, int capacity, const int32_t* ray_dxdy,
             const double* ray_dz, const int32_t* lengths, double hmax, const SolweigSkyLayout* layout,
             const double* band_weights, const uint8_t* sectors, double transmissivity, uint32_t* masks,
             double* planes, float* veg_sums, uint8_t* sky_band_counts, void* work, int64_t work_bytes,
             void* stream) {
    SOLWEIG_CHECK_ARG(dsm && vegdem && vegdem2 && flags && ray_dxdy && ray_dz && lengths && layout &&
                          band_weights && sectors && masks && planes && veg_sums && sky_band_counts,
                      "solweig_svf: null pointer");
    SOLWEIG_CHECK_ARG(rows > 0 && cols > 0 && capacity > 0, "solweig_svf: bad shape");
    SOLWEIG_CHECK_ARG(patches > 0 && patches <= SOLWEIG_MASK_WORDS * 32 && patches == layout->patches,
                      "solweig_svf: %d patches (max %d, layout %d)", patches,
                      SOLWEIG_MASK_WORDS * 32, layout->patches);
    SOLWEIG_CHECK_ARG(layout->nbands > 0 && layout->nbands <= SOLWEIG_MAX_BANDS,
                      "solweig_svf: bad band count %d", layout->nbands);
    const long long pixels = (long long)rows * cols;
    cudaStream_t st = as_stream(stream);
    cudaError_t e = cudaMemsetAsync(masks, 0, sizeof(uint32_t) * 2 * SOLWEIG_MASK_WORDS * pixels, st);
    if (e != cudaSuccess) {
        set_error("solweig_svf: memset: %s", cudaGetErrorString(e));
        return SOLWEIG_ERR_CUDA;
    }
    SvfRayParams rp{rows, cols, patches, capacity, hmax};
    const int words = (patches + 31) / 32;
    const int2* rays = reinterpret_cast<const int2*>(ray_dxdy);
    const float4* g4 = reinterpret_cast<const float4*>(geo32);
    if (!work) {
        dim3 grid(svf_tiles(rows, cols), words);
        if (g4) svf_visibility_kernel<1><<<grid, 32 * kSvfWarps, 0, st>>>(dsm, vegdem, vegdem2, g4, flags, rp, rays,
                                                                          ray_dz, lengths, masks, 0, nullptr, nullptr);
        else svf_visibility_kernel<0><<<grid, 32 * kSvfWarps, 0, st>>>(dsm, vegdem, vegdem2, g4, flags, rp, rays,
                                                                       ray_dz, lengths, masks, 0, nullptr, nullptr);
        SOLWEIG_CHECK_LAUNCH("svf_visibility_kernel");
    } else {
        const SvfWork w = svf_work_layout(rows, cols);
        SOLWEIG_CHECK_ARG(work_bytes >= w.total, "solweig_svf_ex2: work buffer of %lld bytes, need %lld",
                          (long long)work_bytes, w.total);
        SOLWEIG_CHECK_ARG(((uintptr_t)work & 255) == 0, "solweig_svf_ex2: work buffer not 256-byte aligned");
        char* wb = static_cast<char*>(work);
        float* dil = reinterpret_cast<float*>(wb + w.dil);
        float2* ceil = reinterpret_cast<float2*>(wb + w.ceil);
        int* exits = reinterpret_cast<int*>(wb + w.exits);
        // step records when every ray fits kmax (the host's ray tables do)
        longlong2* rec = (g4 && capacity <= w.kmax) ? reinterpret_cast<longlong2*>(wb + w.rec) : nullptr;
        SolweigScene S{};
        S.rows = rows;
        S.cols = cols;
        S.dsm = dsm;
        S.vegdem = vegdem;
        S.vegdem2 = vegdem2;
        S.geo32 = geo32;
        dim3 dgrid(blocks_for(cols, kDilTile), blocks_for(rows, kDilTile));
        if (geo32) ceiling_dilate_kernel<true><<<dgrid, dim3(32, 8), 0, st>>>(S, dil);
        else ceiling_dilate_kernel<false><<<dgrid, dim3(32, 8), 0, st>>>(S, dil);
        SOLWEIG_CHECK_LAUNCH("ceiling_dilate_kernel");
        for (int wd = 0; wd < words; ++wd) {
            const int p0 = wd * kSvfPatchGroup, cnt = std::min(kSvfPatchGroup, patches - p0);
            dim3 cgrid(blocks_for((long long)rows + cols, kCeilLanes), 1, cnt);
            patch_ray_ceiling_kernel<<<cgrid, dim3(kCeilLanes, kCeilWarps), 0, st>>>(S, rays, ray_dz, lengths,
                                                                                     capacity, p0, cnt, dil, ceil);
            SOLWEIG_CHECK_LAUNCH("patch_ray_ceiling_kernel");
            patch_ray_exits_kernel<<<cnt, 1024, 0, st>>>(rows, cols, rays, ray_dz, lengths, capacity, p0, cnt, exits,
                                                          rec, w.kmax);
            SOLWEIG_CHECK_LAUNCH("patch_ray_exits_kernel");
            dim3 grid(svf_tiles(rows, cols), 1);
            if (rec) svf_visibility_warp_kernel<<<blocks_for(svf_tiles(rows, cols), kSvfWarps), 32 * kSvfWarps, 0,
                                                   st>>>(g4, flags, rp, lengths, masks, wd, ceil, exits, rec, w.kmax);
            else if (g4) svf_visibility_kernel<2><<<grid, 32 * kSvfWarps, 0, st>>>(dsm, vegdem, vegdem2, g4, flags,
                                                                                   rp, rays, ray_dz, lengths, masks,
                                                                                   wd, ceil, exits);
            else svf_visibility_kernel<0><<<grid, 32 * kSvfWarps, 0, st>>>(dsm, vegdem, vegdem2, g4, flags, rp,
                                                                           rays, ray_dz, lengths, masks, wd, ceil,
                                                                           nullptr);
            SOLWEIG_CHECK_LAUNCH("svf_visibility_kernel");
        }
    }
    return solweig_svf_reduce(masks, vegdem2, pixels, layout, band_weights, sectors, transmissivity,
                              planes, veg_sums, sky_band_counts, stream);
}

extern "C" int solweig_svf(const double* dsm, const double* vegdem, const double* vegdem2,
                           const uint8_t* flags, int rows, int cols, int patches, int capacity,
                           const int32_t* ray_dxdy, const double* ray_dz, const int32_t* lengths,
                           double hmax, const SolweigSkyLayout* layout,
                           const double* band_weights, const uint8_t* sectors,
                           double transmissivity, uint32_t* masks, double* planes,
                           float* veg_sums, uint8_t* sky_band_counts, void* stream) {
    return solweig_svf_ex(dsm, vegdem, vegdem2, nullptr, flags, rows, cols, patches, capacity, ray_dxdy, ray_dz,
                          lengths, hmax, layout, band_weights, sectors, transmissivity, masks, planes, veg_sums,
                          sky_band_counts, stream);
}

extern "C" int solweig_svf_unpack(const uint32_t* masks, int64_t pixels, int patches, float* shmat,
                                  float* vegmat, float* vbmat, void* stream) {
    SOLWEIG_CHECK_ARG(masks && pixels > 0 && patches > 0 && patches <= SOLWEIG_MASK_WORDS * 32,
                      "solweig_svf_unpack: bad arguments");
    const long long n = (long long)pixels * patches;
    svf_unpack_kernel<<<blocks_for(n, 256), 256, 0, as_stream(stream)>>>(masks, pixels, patches,
                                                                         shmat, vegmat, vbmat);
    SOLWEIG_CHECK_LAUNCH("svf_unpack_kernel");
    return SOLWEIG_OK;
}

extern "C" int solweig_diffsh(const float* shmat, const float* vegshmat, float* diffsh, int64_t n,
                              float transmissivity, void* stream) {
    SOLWEIG_CHECK_ARG(shmat && vegshmat && diffsh && n >= 0, "solweig_diffsh: bad arguments");
    if (n == 0) return SOLWEIG_OK;
    diffsh_kernel<<<blocks_for(n, 256), 256, 0, as_stream(stream)>>>(shmat, vegshmat, diffsh, n,
                                                                     transmissivity);
    SOLWEIG_CHECK_LAUNCH("diffsh_kernel");
    return SOLWEIG_OK;
}
