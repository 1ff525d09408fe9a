// The batched day's shadow sweep on shared-memory windows staged by TMA.
//
// A block sweeps a 16 x 16 pixel tile for one daytime hour.  All rays of the
// hour leave the tile towards the sun, and their offsets grow monotonically,
// so the first steps of every walk stay inside a WIN x WIN pixel window that
// holds the tile in the corner away from the sun (WIN = 48: 32 steps of
// room, 6 blocks per SM; WIN = 40: 24 steps, 8 blocks per SM).  Thread 0
// stages that window of the packed (dsm, canopy, trunk, 0) geometry from HBM
// into shared memory with one cp.async.bulk.tensor load (a 2-D tensor map
// over the raster viewed as rows x (4 * cols) float32) completing on an
// mbarrier.  A walk takes its samples from shared memory up to the step at
// which it leaves the window and from the raster (L1/L2) after it.
//
// No block-wide barrier after the start: while the copy is in flight every
// warp loads its pixels' statics, finds the window exits of its own 8 x 4
// piece (lane-parallel scans) and the window's maximum height M (from the
// day's 16 x 16 tile maxima), then waits on the mbarrier itself and walks.
//
// Warp-vote exit: every 4 steps the lanes of a warp vote (__all_sync) on
// M - dz_{k-1} < dsm_p; once it holds for the whole warp, no sample left in
// the window can change any lane's outputs and the warp jumps to the first
// step outside the window together.
//
// The per-step recurrences are those of shadow_walk_packed (shadow.cuh), in
// the same float64 operations: every output is bit-identical.  The raster
// must carry the packed float32 geometry (SolweigScene::geo32).
#pragma once
#include <cuda.h>

#include "hour.cuh"

namespace solweig {

// Everything lives in an anonymous namespace: each translation unit that
// includes this header instantiates its own copy.
namespace {

constexpr int kSwTile = 16;  // tile side (pixels); also the tile of the height maxima
constexpr int kSwThreads = kSwTile * kSwTile;
constexpr int kSwScanLimit = 256;  // window exits are found by a linear scan up to here
constexpr uint32_t kSwWaitPolls = 1u << 22;

template <int WIN>
struct SweepSmem {
    float4 win[WIN * WIN];  // 128-byte aligned at the start of dynamic shared memory
    unsigned long long bar;
};

// Number of 16 x 16 tiles of the height maxima along each axis.
__host__ __device__ __forceinline__ int sweep_tiles_along(int n) { return (n + kSwTile - 1) / kSwTile; }

// Per 16 x 16 tile, the maximum of the three packed heights (dsm, canopy,
// trunk); one warp per tile row segment, once per day.
__global__ void __launch_bounds__(256) sweep_tile_max_kernel(SolweigScene S, float* __restrict__ tmax) {
    const int ntx = sweep_tiles_along(S.cols), nty = sweep_tiles_along(S.rows);
    const int t = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (t >= ntx * nty) return;
    const int ty = t / ntx, tx = t - ty * ntx;
    const float4* geo = reinterpret_cast<const float4*>(S.geo32);
    float m = 0.f;  // samples outside the raster read as zero
    for (int i = lane; i < kSwTile * kSwTile; i += 32) {
        const int r = ty * kSwTile + i / kSwTile, c = tx * kSwTile + i % kSwTile;
        if (r < S.rows && c < S.cols) {
            const float4 v = __ldg(&geo[(long long)r * S.cols + c]);
            m = fmaxf(m, fmaxf(v.x, fmaxf(v.y, v.z)));
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (lane == 0) tmax[t] = m;
}

__device__ __forceinline__ void sw_mbar_init(unsigned long long* bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"((uint32_t)__cvta_generic_to_shared(bar))
                 : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Arrive on the barrier expecting `bytes` and start the 2-D tile load of the
// box at (x, y) (elements) of `map` into `dst`.  No multicast: the window
// comes from this GPU's own raster into this CTA's shared memory.
__device__ __forceinline__ void sw_tma_load(void* dst, const CUtensorMap* map, int x, int y,
                                            unsigned long long* bar, uint32_t bytes) {
    const uint32_t b = (uint32_t)__cvta_generic_to_shared(bar);
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(b), "r"(bytes) : "memory");
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
            (uint32_t)__cvta_generic_to_shared(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(b)
        : "memory");
}

__device__ __forceinline__ bool sw_mbar_wait(unsigned long long* bar, uint32_t parity, uint32_t limit) {
    const uint32_t a = (uint32_t)__cvta_generic_to_shared(bar);
    for (uint32_t i = 0; i < limit; ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// shadow_walk_packed with the samples of steps [0, kw) read from the window
// (`wbase` = the pixel's own index in it, `wpitch` its row pitch) and the
// warp vote on the window maximum (`wclear`: dz_prev >= wclear means the
// window's maximum minus dz_prev lies below the pixel).  Every lane of the
// warp calls it (lanes without a pixel pass in = false): the window phase
// is a warp-uniform loop so that the vote sees the whole warp.
//
// Samples skipped after a vote all compare below the pixel in every test of
// the walk (building height, canopy top and trunk against dz_k and
// dz_{k-1}), so they would change neither the shadow, the vegetation flags
// nor a canopy top that reaches above the pixel; a canopy top left below the
// pixel does not enter any output.
__device__ __forceinline__ ShadowResult shadow_walk_window(
    bool in, const float4* __restrict__ win, int wpitch, int wbase, int kw, double wclear,
    const float4* __restrict__ geo, int cols, long long p, double a, double top_p, bool bush, double wall,
    const int2* __restrict__ ray, const double* __restrict__ dz, int steps, int kend, double hmax,
    const float2* __restrict__ ceiling) {
    ShadowResult s;
    s.f = a;
    s.topmax = top_p;
    s.shadowed = false;
    s.veg = bush;
    s.ever = false;
    const bool is_wall = wall > 0.0;
    const bool nonneg = a >= 0.0;
    const double pinf = __longlong_as_double(0x7ff0000000000000ll);
    const double clear = nonneg ? nextafter(hmax - a, pinf) : pinf;
    double dz_prev = 0.0;
    bool final = false;
    auto step = [&](const float4 v, double dzk) -> bool {  // true: the walk is over
        s.f = fmax(s.f, (double)v.x - dzk);
        s.shadowed = s.f > a;
        if (v.y <= 0.f && v.z <= 0.f && nonneg && s.topmax >= 0.0) {
            if (s.shadowed) s.veg = false;
            else s.ever = s.ever || s.veg;
        } else {
            const double tq = v.y, bq = v.z;
            s.topmax = fmax(s.topmax, tq - dzk);
            if (s.shadowed) {
                s.veg = false;
            } else {
                const int n = (int)(tq - dzk > a) + (int)(bq - dzk > a) + (int)(tq - dz_prev > a) +
                              (int)(bq - dz_prev > a);
                s.veg = s.veg || (n > 0 && n < 4);
                s.ever = s.ever || s.veg;
            }
        }
        return s.shadowed && (!is_wall || s.f - a >= wall);
    };
    // true: nothing further can change (the exits of shadow_walk_packed)
    auto settled = [&](long long q, int k, double dzk) {
        if (dz_prev >= clear && (!is_wall || (s.topmax >= 0.0 && hmax - dzk <= s.topmax))) return true;
        if (ceiling != nullptr && k >= 4 && (k & 3) == 0) {
            const double e = __dsub_ru((double)__ldg(&ceiling[q]).x, dz_prev);
            if (nonneg && e < a && (!is_wall || (s.topmax >= 0.0 && e <= s.topmax))) return true;
        }
        return false;
    };
    // phase 1: samples from the window, the warp stepping together
    bool active = in && kw > 0;
    int k = 0;
    const int kwm = __reduce_max_sync(0xffffffffu, active ? kw : 0);
    for (int kk = 0; kk < kwm; ++kk) {
        if (kk >= 4 && (kk & 3) == 0 && __all_sync(0xffffffffu, !active || (nonneg && dz_prev >= wclear)))
            break;  // no window sample left can reach above any lane's pixel
        if (active) {
            if (kk >= kw) {
                active = false;
            } else {
                const int2 o = __ldg(&ray[kk]);
                const double dzk = __ldg(&dz[kk]);
                if (settled(p + (long long)o.x * cols + o.y, kk, dzk) || step(win[wbase + o.x * wpitch + o.y], dzk)) {
                    final = true;
                    active = false;
                } else {
                    dz_prev = dzk;
                    k = kk + 1;
                }
            }
        }
    }
    if (in && !final) {
        // samples skipped by the vote all lie below the pixel: resume at the
        // first step outside the window, with dz_prev of the step before it
        if (k < kw) {
            k = kw;
            dz_prev = __ldg(&dz[k - 1]);
        }
        // phase 2: samples from the raster
        for (; k < kend; ++k) {
            const int2 o = __ldg(&ray[k]);
            const double dzk = __ldg(&dz[k]);
            const long long q = p + (long long)o.x * cols + o.y;
            if (settled(q, k, dzk) || step(__ldg(&geo[q]), dzk)) {
                final = true;
                break;
            }
            dz_prev = dzk;
        }
        if (!final && k < steps) {
            // First step whose sample is outside the raster: all shifted values are 0.
            s.f = fmax(s.f, 0.0);
            s.shadowed = s.f > a;
            s.topmax = fmax(s.topmax, 0.0);
            if (s.shadowed) s.veg = false;
            s.ever = s.ever || s.veg;
        }
    }
    return s;
}

// Quad epilogue of shadow_quad_pixel for a walk result (no water here).
__device__ __forceinline__ void write_quad(const SolweigScene& S, const SolweigHour& h, long long p, double a,
                                           double wall, uint8_t fl, const ShadowResult& s,
                                           float4* __restrict__ quad) {
    quad[p] = quad_from_walk(S, h, p, a, wall, fl, s, nullptr);
}

// grid (tiles along columns, tiles along rows, hours of the range); kSwThreads
// threads; dynamic shared memory sweep_smem_bytes<WIN>().  Scenes with water
// use the raster sweep kernel (they also need the first direction's Lup).
// `hours`, `quads`, `ceiling` (planes [hour][px]) and `exits` ([hour][rows +
// cols]) point at the range's first hour; grid.z indexes the hours of the
// range.  `tmax`: the day's 16 x 16 tile maxima (sweep_tile_max_kernel).
template <int WIN>
__global__ void __launch_bounds__(kSwThreads, WIN <= 40 ? 8 : 6)
    day_sweep_tma_kernel(const __grid_constant__ CUtensorMap geo_map, SolweigScene S,
                         const SolweigHour* __restrict__ hours, float4* __restrict__ quads,
                         const float2* __restrict__ ceiling, const int* __restrict__ exits,
                         const float* __restrict__ tmax, int* __restrict__ error) {
    static_assert(WIN >= kSwTile && WIN <= 64, "window side");
    const SolweigHour& h = hours[blockIdx.z];
    if (!h.daytime) return;
    extern __shared__ unsigned char sw_raw[];
    SweepSmem<WIN>& sm = *reinterpret_cast<SweepSmem<WIN>*>(
        (reinterpret_cast<uintptr_t>(sw_raw) + 127) & ~static_cast<uintptr_t>(127));
    const int tid = threadIdx.x;
    const int2* ray = reinterpret_cast<const int2*>(h.ray_dxdy);
    const int K = h.steps;
    const int r0 = blockIdx.y * kSwTile, c0 = blockIdx.x * kSwTile;
    // the window holds the tile in its corner away from the sun
    const int2 last = K > 0 ? __ldg(&ray[K - 1]) : make_int2(0, 0);
    const int wr0 = last.x < 0 ? r0 + kSwTile - WIN : r0;
    const int wc0 = last.y < 0 ? c0 + kSwTile - WIN : c0;
    if (tid == 0) sw_mbar_init(&sm.bar);
    __syncthreads();  // the barrier is initialised before anyone polls it
    if (tid == 0) sw_tma_load(sm.win, &geo_map, 4 * wc0, wr0, &sm.bar, (uint32_t)(WIN * WIN * 16));

    // this thread's pixel: warps take 8 x 4 (columns x rows) pieces
    const int w = tid >> 5, l = tid & 31;
    const int tx0 = (w & 1) * 8, ty0 = (w >> 1) * 4;
    const int tx = tx0 + (l & 7), ty = ty0 + (l >> 3);
    const int r = r0 + ty, c = c0 + tx;
    const bool in = r < S.rows && c < S.cols;
    const long long npx = (long long)S.rows * S.cols;
    const long long p = in ? (long long)r * S.cols + c : 0;
    const double a = in ? S.dsm[p] : 0.0;
    const double wall = in ? S.walls[p] : 0.0;
    const uint8_t fl = in ? S.flags[p] : 0;
    const double top_p = in ? S.vegdem[p] : 0.0;
    // this hour's ray exits and ceiling plane
    const int* ex = exits + (long long)blockIdx.z * (S.rows + S.cols);
    const float2* ceil_h = ceiling ? ceiling + (long long)blockIdx.z * npx : nullptr;
    int kend = 0;
    if (in) kend = min(K, min(__ldg(&ex[r]), __ldg(&ex[S.rows + c])));

    // window exits of the piece: lanes 0-3 scan its rows, lanes 4-11 its
    // columns (linear scans, capped: a smaller value only moves samples to
    // the raster path)
    int scan = 0;
    if (l < 12) {
        const bool row = l < 4;
        const int pos = row ? r0 + ty0 + l - wr0 : c0 + tx0 + (l - 4) - wc0;
        const int lim = K < kSwScanLimit ? K : kSwScanLimit;
        for (; scan < lim; ++scan) {
            const int2 o = __ldg(&ray[scan]);
            const int v = pos + (row ? o.x : o.y);
            if (v < 0 || v >= WIN) break;
        }
    }
    const int row_exit = __shfl_sync(0xffffffffu, scan, l >> 3);
    const int col_exit = __shfl_sync(0xffffffffu, scan, 4 + (l & 7));
    // the window's maximum height, from the tile maxima it overlaps (tiles
    // outside the raster count as zero, as the copy fills them)
    float m = 0.f;
    {
        const int ntx = sweep_tiles_along(S.cols), nty = sweep_tiles_along(S.rows);
        const int ya = wr0 >> 4, yb = (wr0 + WIN - 1) >> 4;  // arithmetic shifts: floor
        const int xa = wc0 >> 4, xb = (wc0 + WIN - 1) >> 4;
        const int tyi = ya + (l >> 2), txi = xa + (l & 3);
        if (l < 16 && tyi <= yb && txi <= xb && tyi >= 0 && tyi < nty && txi >= 0 && txi < ntx)
            m = __ldg(&tmax[tyi * ntx + txi]);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    }
    // wait for the window (bounded, every thread); on a timeout record the
    // error, wait once more for the copy in flight and walk from the raster
    const bool got = sw_mbar_wait(&sm.bar, 0, kSwWaitPolls);
    if (!got) sw_mbar_wait(&sm.bar, 0, kSwWaitPolls);
    const bool staged = __all_sync(0xffffffffu, got);
    if (!staged && l == 0) raise_day_flag(error, 2);
    const int kw = staged && in ? min(kend, min(row_exit, col_exit)) : 0;
    const double pinf = __longlong_as_double(0x7ff0000000000000ll);
    const double wclear = a >= 0.0 ? nextafter((double)m - a, pinf) : pinf;
    const ShadowResult s = shadow_walk_window(in, sm.win, WIN, (r - wr0) * WIN + (c - wc0), kw, wclear,
                                              reinterpret_cast<const float4*>(S.geo32), S.cols, p, a, top_p,
                                              (fl & 2) != 0, wall, ray, h.ray_dz, K, kend, S.hmax, ceil_h);
    if (in) write_quad(S, h, p, a, wall, fl, s, quads + (long long)blockIdx.z * npx);
}

// Tensor map of the packed geometry viewed as a rows x (4 * cols) float32
// array, box WIN rows x 4 * WIN floats (one window); elements outside the
// raster read as zero (the walks never use them: they stop at the raster
// edge).  The x coordinate of a window is 4 * its first column, so every
// copy starts on a 16-byte boundary.  The driver's encoder is looked up once
// through the runtime.
inline int sweep_geo_map(const SolweigScene& S, int win, CUtensorMap* map) {
    using Encode = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
    static Encode encode = nullptr;
    static int looked_up = 0;
    if (!looked_up) {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        const cudaError_t e = cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &fn, 12000,
                                                               cudaEnableDefault, &q);
        if (e == cudaSuccess && q == cudaDriverEntryPointSuccess) encode = reinterpret_cast<Encode>(fn);
        looked_up = 1;
    }
    SOLWEIG_CHECK_ARG(encode != nullptr, "day sweep: cuTensorMapEncodeTiled is not available");
    SOLWEIG_CHECK_ARG(S.geo32 && ((uintptr_t)S.geo32 & 15) == 0, "day sweep: packed geometry missing or unaligned");
    const cuuint64_t dims[2] = {4ull * (cuuint64_t)S.cols, (cuuint64_t)S.rows};
    const cuuint64_t strides[1] = {16ull * (cuuint64_t)S.cols};
    const cuuint32_t box[2] = {4u * (cuuint32_t)win, (cuuint32_t)win};
    const cuuint32_t estr[2] = {1u, 1u};
    const CUresult r = encode(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<void*>(S.geo32), dims, strides,
                              box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                              CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        set_error("day sweep: cuTensorMapEncodeTiled failed (%d)", (int)r);
        return SOLWEIG_ERR_CUDA;
    }
    return SOLWEIG_OK;
}

template <int WIN>
inline size_t sweep_smem_bytes() {
    return sizeof(SweepSmem<WIN>) + 128;
}

}  // namespace

}  // namespace solweig
