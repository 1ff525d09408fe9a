// Kernels and launch helpers of the batched day, shared by the batched
// entry points (day.cu) and the day gradient (adjoint.cu).  Everything lives
// in an anonymous namespace: each translation unit instantiates its own copy.
#pragma once
#include <cuda_bf16.h>

#include "ceiling.cuh"
#include "gvf_fields.cuh"
#include "hour.cuh"
#include "radiation.cuh"
#include "sweep_tma.cuh"
#include "tcgen05.cuh"

namespace solweig {

namespace {

constexpr int kDayBX = 32, kDayBY = 8;
constexpr int kK = SOLWEIG_MAX_PATCHES;   // contraction depth (patches, padded)
constexpr int kSBO = (kK / 8) * 128;      // bytes between 8-row groups of an operand
constexpr int kARows = 128;               // pixels per contraction tile (MMA M)
constexpr int kABytes = kARows * kK * 2;  // one A operand in shared memory
constexpr int kMaxDayHours = 64;
constexpr uint32_t kWaitPolls = 1u << 24;

// Element offset of (row n, patch k) in the canonical K-major layout.
__host__ __device__ __forceinline__ int canon_off(int n, int k) {
    return (n >> 3) * (kSBO / 2) + (k >> 3) * 64 + (n & 7) * 8 + (k & 7);
}

// Sunlit / shaded tables of one hour (size a multiple of 16 bytes).
struct DayTable {
    double tsun[kK];        // sorted: patch sunlit  <=> tan(asvf) <  T_k
    double vshade[kK];      // sorted: patch shaded  <=> tan(asvf) >= V_k
    uint32_t suf[kK + 1][SOLWEIG_MASK_WORDS];  // patches at sorted sunlit positions >= i
    uint32_t pre[kK + 1][SOLWEIG_MASK_WORDS];  // patches at sorted shaded positions <  j
    uint32_t test[SOLWEIG_MASK_WORDS];         // longwave sun test of the hour
    uint32_t pad[5];
    // first sorted position whose threshold is >= bucket boundary i (see
    // tan_bucket): the counts of thresholds <= t start there for t in bucket i
    uint8_t sun_start[256];
    uint8_t shd_start[256];
    // hour scalars of the radiation loop, rounded once from the float64 plan
    float band_down[SOLWEIG_MAX_BANDS], band_side[SOLWEIG_MAX_BANDS];
    float lw_shade, lw_sun, sw_shade, sw_sun, rad_d, rad_g, direct_up, rad_i_sin, rad_i_cos, rad_ratio;
    float wave_w, tan_zen, night_lup, night_lup_water;
    float pad2[2];
};

// 256 buckets of tan(asvf): boundary i = tan(i * pi / 512) for i >= 1,
// -inf for i = 0 (the same float64 expression wherever it is evaluated).
__device__ __forceinline__ double tan_bucket_bound(int i) {
    return i == 0 ? __longlong_as_double(0xfff0000000000000ll) : tan((double)i * (kPi / 512.0));
}

// Largest i with tan_bucket_bound(i) <= t.
__device__ __forceinline__ int tan_bucket(double t) {
    int i = (int)(atan(t) * (512.0 / kPi));
    i = i < 0 ? 0 : (i > 255 ? 255 : i);
    while (i < 255 && tan_bucket_bound(i + 1) <= t) ++i;
    while (i > 0 && tan_bucket_bound(i) > t) --i;
    return i;
}

// Number of entries of the ascending a[0..n) that are <= t, starting from
// `from` = the number of entries below the bucket boundary of t.
__device__ __forceinline__ int count_le_from(const double* a, int n, int from, double t) {
    int i = from;
    while (i < n && a[i] <= t) ++i;
    return i;
}
static_assert(sizeof(DayTable) % 16 == 0, "DayTable must be a multiple of 16 bytes");

// Band boundaries (patch index) of the sky layouts the batched form supports.
template <int OPT>
struct Bands;
template <>
struct Bands<2> {  // 153 patches: 31, 30, 28, 24, 19, 13, 7, 1
    __host__ __device__ static constexpr int off(int b) {
        return b <= 0 ? 0 : b == 1 ? 31 : b == 2 ? 61 : b == 3 ? 89 : b == 4 ? 113 : b == 5 ? 132
               : b == 6 ? 145 : b == 7 ? 152 : 153;
    }
};
template <>
struct Bands<1> {  // 145 patches: 30, 30, 24, 24, 18, 12, 6, 1
    __host__ __device__ static constexpr int off(int b) {
        return b <= 0 ? 0 : b == 1 ? 30 : b == 2 ? 60 : b == 3 ? 84 : b == 4 ? 108 : b == 5 ? 126
               : b == 6 ? 138 : b == 7 ? 144 : 145;
    }
};

// sum over bands of w[b] * popcount(m restricted to band b).
template <int OPT>
__device__ __forceinline__ float band_weighted(const uint32_t (&m)[SOLWEIG_MASK_WORDS], const float* w) {
    float s = 0.f;
#pragma unroll
    for (int b = 0; b < 8; ++b) {
        const int lo = Bands<OPT>::off(b), hi = Bands<OPT>::off(b + 1);
        int c = 0;
#pragma unroll
        for (int wd = 0; wd < SOLWEIG_MASK_WORDS; ++wd) {
            const int a = lo > wd * 32 ? lo : wd * 32;
            const int e = hi < wd * 32 + 32 ? hi : wd * 32 + 32;
            if (a < e) {
                const uint32_t mask = (e - a == 32) ? 0xffffffffu : (((1u << (e - a)) - 1u) << (a - wd * 32));
                c += __popc(m[wd] & mask);
            }
        }
        s = fmaf((float)c, w[b], s);
    }
    return s;
}

// Patches of m in each band (popcounts of the band's bit ranges), and the
// weighted sum of such counts.
template <int OPT>
__device__ __forceinline__ void band_counts(const uint32_t (&m)[SOLWEIG_MASK_WORDS], float (&c)[8]) {
#pragma unroll
    for (int b = 0; b < 8; ++b) {
        const int lo = Bands<OPT>::off(b), hi = Bands<OPT>::off(b + 1);
        int n = 0;
#pragma unroll
        for (int wd = 0; wd < SOLWEIG_MASK_WORDS; ++wd) {
            const int a = lo > wd * 32 ? lo : wd * 32;
            const int e = hi < wd * 32 + 32 ? hi : wd * 32 + 32;
            if (a < e) {
                const uint32_t mask = (e - a == 32) ? 0xffffffffu : (((1u << (e - a)) - 1u) << (a - wd * 32));
                n += __popc(m[wd] & mask);
            }
        }
        c[b] = (float)n;
    }
}
__device__ __forceinline__ float band_dot(const float (&c)[8], const float* w) {
    float s = 0.f;
#pragma unroll
    for (int b = 0; b < 8; ++b) s = fmaf(c[b], w[b], s);
    return s;
}

// Number of entries of the ascending array a[0..n) that are <= t.
__device__ __forceinline__ int count_le(const double* a, int n, double t) {
    int lo = 0;
    while (n > 0) {
        const int half = n >> 1;
        if (a[lo + half] <= t) {
            lo += half + 1;
            n -= half + 1;
        } else {
            n = half;
        }
    }
    return lo;
}

// Monotone integer keys of the doubles (NaN excluded).
__device__ __forceinline__ unsigned long long dkey(double x) {
    const unsigned long long u = (unsigned long long)__double_as_longlong(x);
    return (u >> 63) ? ~u : (u | 0x8000000000000000ull);
}
__device__ __forceinline__ double dval(unsigned long long k) {
    const unsigned long long u = (k >> 63) ? (k & 0x7fffffffffffffffull) : ~k;
    return __longlong_as_double((long long)u);
}

// Smallest double t in [-inf, +inf] with pred(t) true, for pred monotone
// (false, then true); +inf when pred is false for every finite t.
template <typename Pred>
__device__ double first_true(Pred pred) {
    const double ninf = __longlong_as_double(0xfff0000000000000ll);
    const double pinf = __longlong_as_double(0x7ff0000000000000ll);
    if (pred(ninf)) return ninf;
    if (!pred(pinf)) return pinf;
    unsigned long long lo = dkey(ninf), hi = dkey(pinf);  // pred(lo) false, pred(hi) true
    while (hi - lo > 1) {
        const unsigned long long mid = lo + (hi - lo) / 2;
        if (pred(dval(mid))) hi = mid;
        else lo = mid;
    }
    return dval(hi);
}

// ---------------------------------------------------------------- kernels 1, 2

// Pixel of this thread in a block tile of bx x by pixels.  When the tile
// holds whole 8 x 4 (columns x rows) pieces, each warp takes one such piece
// instead of 32 pixels of one row: walk lengths of nearby pixels are alike in
// both directions, so the warp's longest walk is closer to its mean (30%
// fewer warp steps on the synthetic city); a warp's loads still cover 4 rows
// of 32-128 contiguous bytes, as many sectors as one row of 32 pixels.
__device__ __forceinline__ void warp_tile_pixel(int bx, int by, int& r, int& c) {
    if (bx % 8 == 0 && by % 4 == 0) {
        const int t = threadIdx.y * bx + threadIdx.x, w = t >> 5, l = t & 31;
        const int wx = w % (bx / 8), wy = w / (bx / 8);
        c = blockIdx.x * bx + wx * 8 + (l & 7);
        r = blockIdx.y * by + wy * 4 + (l >> 3);
    } else {
        c = blockIdx.x * bx + threadIdx.x;
        r = blockIdx.y * by + threadIdx.y;
    }
}

// REC: the walks read the hour's step records (rec + z * kmax, written by
// day_ray_exits_kernel) instead of the (dx, dy) and dz tables.  40 registers
// (6 blocks of 256 per SM): the walk's float64 state no longer spills (per
// 2000^2 day 5.77 ms against 5.97 ms at 32 registers and 8 blocks).
template <bool REC>
__global__ void __launch_bounds__(256, 6) day_shadow_kernel(SolweigScene S,
                                                                   const SolweigHour* __restrict__ hours,
                                                                   float4* __restrict__ quads,
                                                                   float* __restrict__ lup_first,
                                                                   const float2* __restrict__ ceiling,
                                                                   const int* __restrict__ exits,
                                                                   const longlong2* __restrict__ rec, int kmax) {
    const int z = blockIdx.z;
    const SolweigHour& h = hours[z];
    if (!h.daytime) return;
    int r, c;
    warp_tile_pixel(blockDim.x, blockDim.y, r, c);
    const bool in = r < S.rows && c < S.cols;
    const long long n = (long long)S.rows * S.cols;
    if (!in) return;
    shadow_quad_pixel<REC>(S, h, r, c, quads + z * n, lup_first ? lup_first + z * n : nullptr,
                           ceiling ? ceiling + z * n : nullptr,
                           exits ? exits + (long long)z * (S.rows + S.cols) : nullptr,
                           REC ? rec + (long long)z * kmax : nullptr);
}

// Per daytime hour, the first-outside step of every row and column of the
// raster (first_outside), for the bounds-check-free sweep, and with rec the
// hour's step records for the steps [0, min(steps, kmax)).  A monotone ray
// leaves the raster within max(rows, cols) steps, so kmax = max(rows, cols)
// + 2 covers every walk; a ray table that stays inside longer has its exits
// cut to kmax and sets the error flag to 3 (that hour's results invalid).
__global__ void __launch_bounds__(1024) day_ray_exits_kernel(SolweigScene S, const SolweigHour* __restrict__ hours,
                                                             int* __restrict__ exits, longlong2* __restrict__ rec,
                                                             int kmax, int* __restrict__ error) {
    const SolweigHour& h = hours[blockIdx.x];
    if (!h.daytime) return;
    int* ex = exits + (long long)blockIdx.x * (S.rows + S.cols);
    ray_exits_block(reinterpret_cast<const int2*>(h.ray_dxdy), h.steps, S.rows, S.cols, ex);
    if (rec == nullptr) return;
    const int K = min(h.steps, kmax);
    ray_records_block(reinterpret_cast<const int2*>(h.ray_dxdy), h.ray_dz, K, S.cols,
                      rec + (long long)blockIdx.x * kmax);
    if (h.steps <= kmax) return;
    __syncthreads();  // ex[] written by the whole block
    int cut = 0;
    for (int i = threadIdx.x; i < S.rows + S.cols; i += blockDim.x) {
        if (ex[i] > kmax) {
            ex[i] = kmax;
            cut = 1;
        }
    }
    if (cut) raise_day_flag(error, 3);
}

struct DayGvfArgs {
    int first, second, halo;
};

// Tiles of the hour-vectorized GVF kernel: 32 x 32 pixels, halo 21 (the 1 m
// walk, second = 22).  A tile is interior when its halo lies inside the raster.
constexpr int kHvTile = 32, kHvHalo = 21, kHvPitch = kHvTile + 2 * kHvHalo;
static_assert(kHvTile == 32, "the hour-vectorized GVF maps its 32 warps to 8 x 4 pieces of a 32 x 32 tile");

__host__ __device__ __forceinline__ bool hv_tile_interior(int rows, int cols, int tr, int tc) {
    const int row0 = tr * kHvTile - kHvHalo, col0 = tc * kHvTile - kHvHalo;
    return row0 >= 0 && col0 >= 0 && row0 + kHvPitch <= rows && col0 + kHvPitch <= cols;
}

// gvf[z][0] = Lup GVF (ambient added), gvf[z][1] = albedo GVF, gvf[z][2] = shadow.
// nosh = albedo-without-shadow GVF: the same for every hour (walk geometry and
// albedo only), so every daytime launch writes the same values.
template <int TY, int FIRST, int SECOND, int TABLE, bool WATER>
__global__ void __launch_bounds__(32 * TY) day_gvf_kernel(SolweigScene S, const SolweigHour* __restrict__ hours,
                                                         DayGvfArgs ga, GvfTable<TABLE> tab,
                                                         const float4* __restrict__ quads,
                                                         const float* __restrict__ lup_first_all,
                                                         float* __restrict__ gvf, float* __restrict__ nosh) {
    const int z = blockIdx.z;
    const SolweigHour& h = hours[z];
    if (!h.daytime) return;
    const int bx = blockIdx.x, by = blockIdx.y;
    const long long n = (long long)S.rows * S.cols;
    const float4* quad = quads + z * n;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int H = ga.halo, second = ga.second, first = ga.first;
    const int pitch = 32 + 2 * H;
    float4* tile = reinterpret_cast<float4*>(smem_raw);
    const int row0 = by * TY - H, col0 = bx * 32 - H;
    load_quad_tile(tile, pitch, TY + 2 * H, quad, S.rows, S.cols, row0, col0);
    __syncthreads();
    const int c = bx * 32 + threadIdx.x;
    const int r = by * TY + threadIdx.y;
    if (r >= S.rows || c >= S.cols) return;
    const long long p = (long long)r * S.cols + c;
    const float4* own_cell = tile + (threadIdx.y + H) * pitch + threadIdx.x + H;
    const float4 own = *own_cell;
    const double ta = h.ta;
    const float lwall = (float)(kSBC * 0.9 * pow4(h.tgwall + ta + 273.15) - kSBC * 0.9 * pow4(ta + 273.15));
    const float albedo_b = 0.2f;
    const uint32_t face = S.gvf_face[p];
    const bool own_ground = (__float_as_int(own.w) & kQuadGround) != 0;
    float lup, alb, nsh;
    if (WATER) {
        const float* lfp = lup_first_all + z * n;
        GvfScalars gs{lwall, albedo_b, first, second};
        auto sample = [&](int rr, int cc) -> float4 { return tile[(rr - row0) * pitch + (cc - col0)]; };
        auto lfirst = [&](int rr, int cc) -> float { return __ldg(&lfp[(long long)rr * S.cols + cc]); };
        const GvfSums g = gvf_walk(sample, lfirst, true, r, c, S.rows, S.cols, tab.offs, face, own, gs);
        lup = g.lup[0];
        alb = g.alb[0];
        nsh = g.nosh[0];
    } else {
        lup = alb = nsh = 0.f;
        const bool interior = row0 >= 0 && col0 >= 0 && row0 + TY + 2 * H <= S.rows && col0 + pitch <= S.cols;
        const float inv_first = 1.f / first, inv_first1 = 1.f / (first + 1);
        const float inv_second = 1.f / second, inv_second1 = 1.f / (second + 1);
#pragma unroll 1
        for (int j = 0; j < SOLWEIG_GVF_DIRECTIONS; ++j) {
            const bool fj = (face >> j) & 1u;
            const int base = j * (SECOND > 0 ? SECOND : second);
            GvfDir d;
            if (SECOND > 0) {
                d = interior ? gvf_direction_fixed<true, FIRST, SECOND>(own_cell, tab.delta + base, tab.offs + base, r,
                                                                        c, S.rows, S.cols, own_ground, lwall,
                                                                        albedo_b, fj)
                             : gvf_direction_fixed<false, FIRST, SECOND>(own_cell, tab.delta + base, tab.offs + base,
                                                                         r, c, S.rows, S.cols, own_ground, lwall,
                                                                         albedo_b, fj);
            } else {
                d = interior ? gvf_direction<true>(own_cell, tab.delta + base, tab.offs + base, r, c, S.rows, S.cols,
                                                   own_ground, first, second, inv_first, inv_first1, inv_second,
                                                   inv_second1, lwall, albedo_b, fj)
                             : gvf_direction<false>(own_cell, tab.delta + base, tab.offs + base, r, c, S.rows, S.cols,
                                                    own_ground, first, second, inv_first, inv_first1, inv_second,
                                                    inv_second1, lwall, albedo_b, fj);
            }
            lup += d.lup;
            alb += d.alb;
            nsh += d.nosh;
        }
        const float ob = own_ground ? 1.f : 0.f;
        nsh *= ob;
        lup += 18.f * (own.y * (1.f - ob));
        alb += 18.f * (own.z * (1.f - ob) * own.x);
        nsh += 18.f * (own.z * (1.f - ob));
    }
    const double ambient = kSBC * (double)S.emis[p] * pow4(ta + 273.15);
    gvf[(3 * z) * n + p] = (float)((double)(lup / 18.f) + ambient);
    gvf[(3 * z + 1) * n + p] = alb / 18.f;
    gvf[(3 * z + 2) * n + p] = own.x;
    nosh[p] = nsh / 18.f;
}

// Hour-vectorized GVF for interior 32 x 32 tiles (the 1 m walk: first = 1,
// second = 22), all daytime hours of the day in one block.  The walk length
// of every direction (first building step) and the albedo-without-shadow
// plane depend only on the ground bits and the albedo, so they are computed
// once; then per pass of kHvCh daytime hours the tile is staged as
// (Lup, albedo*shadow) pairs plus the sunlit-wall bits of those hours, and
// every walked sample is one pair of 16-byte shared loads serving all kHvCh
// hours.  The sunlit-wall statistics need only the first step at which each
// hour's bit appears: seen at step f < hit means n_sun = second - f (the
// steps after a building hit keep counting, as in gvf_direction_fixed).
// Same recurrences as gvf_direction_fixed and the same float32 sums along
// the walk, except albedo*shadow, which is rounded once per sample here
// instead of fused into the sum; the per-direction weights are applied as
// fused multiply-adds (a few ulp from the per-hour kernel's order).
//
// Border tiles (halo reaching outside the raster) stage zeros outside and
// follow the per-hour walk's edge rule: a walk whose first step leaves the
// raster sees no ground (hit = 0); one that leaves at step L > 0 repeats its
// last sample (step L - 1) for the remaining second - L steps and never hits.
// Per direction the kernel keeps `lim` (samples read) and a frozen-tail bit
// (then hit = second, else hit = lim): 6 bits, 5 directions per word.
//
// Shared memory: the two (Lup, albedo*shadow) float4 planes, one byte per
// pixel of bits (ground during the walk-length pass, then the pass hours'
// sunlit-wall bits 0..3) and the daytime hour list; the albedo of the
// walk-length pass lives in the second float4 plane before the first hour
// pass overwrites it.  A warp's byte loads (8 x 4 pixels, rows 74 bytes
// apart) touch distinct banks: one wavefront.
constexpr int kHvN = kHvPitch * kHvPitch;
constexpr int kHvCh = 4;
constexpr int kHvThreads = kHvTile * kHvTile;
constexpr int kHvBitsBytes = (kHvN + 15) & ~15;

size_t hv_smem_bytes() { return (size_t)kHvN * 2 * sizeof(float4) + kHvBitsBytes + 64 * sizeof(int); }

// The hour-independent part of the hour-vectorized GVF for the pixel at tile
// offset `own` (tile staged with its ground bits and albedo): the walk-length
// code of every direction (5 per word: lim, frozen-tail bit) and the
// albedo-without-shadow GVF sum (before / 18).  Shared by day_gvf_hv_kernel
// and gvf_statics_kernel.
__device__ __forceinline__ float hv_static_walks(const uint8_t* bits, const float* albs, int own, bool own_ground,
                                                 bool interior, int r, int c, int rows, int cols,
                                                 const GvfTable<22>& tab, uint32_t (&hits)[4]) {
    constexpr int FIRST = 1, SECOND = 22;
    constexpr float albedo_b = 0.2f;
    constexpr float inv_first = 1.f / FIRST, inv_first1 = 1.f / (FIRST + 1);
    constexpr float inv_second = 1.f / SECOND;
    const float ob = own_ground ? 1.f : 0.f;
    float nsh = 0.f;
#pragma unroll
    for (int w = 0; w < 4; ++w) hits[w] = 0u;
    for (int j = 0; j < SOLWEIG_GVF_DIRECTIONS; ++j) {
        int hit = 0, lim = 0;
        float s_alb = 0.f, n_alb = 0.f;
        if (own_ground) {
            hit = lim = SECOND;
            for (int m = 0; m < SECOND; ++m) {
                if (!interior) {
                    const int2 o = tab.offs[j * SECOND + m];
                    if (!in_raster(r + o.x, c + o.y, rows, cols)) {
                        if (m == 0) {
                            hit = lim = 0;
                        } else {  // frozen tail: step m and the rest repeat step m - 1
                            lim = m;
                            const float al = albs[own + tab.delta[j * SECOND + m - 1]];
                            s_alb += al;
                            s_alb += (SECOND - 1 - m) * al;
                        }
                        break;
                    }
                }
                const int off = own + tab.delta[j * SECOND + m];
                if (!(bits[off] & 1u)) {
                    hit = lim = m;
                    break;
                }
                s_alb += albs[off];
                if (m + 1 == FIRST) n_alb = s_alb;
            }
        }
        hits[j / 5] |= ((uint32_t)lim | (hit > lim ? 32u : 0u)) << (6 * (j % 5));
        const int n_wall = SECOND - hit;
        const int n_wall_first = FIRST > hit ? FIRST - hit : 0;
        const float nosh1 = n_wall_first > 0 ? ((float)n_wall_first * albedo_b + n_alb) * inv_first1 : n_alb * inv_first;
        const float nosh2 = n_wall > 0 ? ((float)n_wall * albedo_b + s_alb) * inv_second : s_alb * inv_second;
        nsh += (nosh1 * 0.5f + nosh2 * 0.4f) * (1.f / 0.9f);
    }
    nsh *= ob;
    nsh += 18.f * (albs[own] * (1.f - ob));
    return nsh;
}

__global__ void __launch_bounds__(kHvThreads, 1) day_gvf_hv_kernel(SolweigScene S, const SolweigHour* __restrict__ hours,
                                                                  int nhours, GvfTable<22> tab,
                                                                  const float4* __restrict__ quads,
                                                                  float* __restrict__ gvf, float* __restrict__ nosh) {
    constexpr int FIRST = 1, SECOND = 22;
    const int tr = blockIdx.y, tc = blockIdx.x;
    const bool interior = hv_tile_interior(S.rows, S.cols, tr, tc);
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float4* LA = reinterpret_cast<float4*>(smem_raw);  // Lup, albsh of pass hours 0, 1
    float4* LB = LA + kHvN;                            // pass hours 2, 3
    uint8_t* bits = reinterpret_cast<uint8_t*>(LB + kHvN);    // ground bit, then sunlit-wall bits
    float* albs = reinterpret_cast<float*>(LB);                // albedo (walk-length pass only)
    int* dayh = reinterpret_cast<int*>(bits + kHvBitsBytes);   // daytime hour indices
    __shared__ int nday;
    const int tid = threadIdx.y * kHvTile + threadIdx.x;
    const long long n = (long long)S.rows * S.cols;
    const int row0 = tr * kHvTile - kHvHalo, col0 = tc * kHvTile - kHvHalo;
    if (tid == 0) {
        int k = 0;
        for (int h = 0; h < nhours && k < 64; ++h)
            if (hours[h].daytime) dayh[k++] = h;
        nday = k;
    }
    __syncthreads();
    const int nd = nday;
    if (nd == 0) return;
    const bool statics = S.gvf_hits != nullptr && S.gvf_nosh != nullptr;
    if (!statics) {
        const float4* q0 = quads + (long long)dayh[0] * n;
        for (int i = tid; i < kHvN; i += kHvThreads) {
            const int rr = row0 + i / kHvPitch, cc = col0 + i % kHvPitch;
            const bool in = interior || in_raster(rr, cc, S.rows, S.cols);
            const float4 q = in ? q0[(long long)rr * S.cols + cc] : make_float4(0.f, 0.f, 0.f, 0.f);
            bits[i] = (uint8_t)(__float_as_int(q.w) & kQuadGround);
            albs[i] = q.z;
        }
        __syncthreads();
    }
    // each warp walks an 8 x 4 (columns x rows) piece of the tile: walk lengths
    // of nearby pixels are alike in both directions (24% fewer warp steps than
    // a row of 32 on the synthetic city), and a warp's shared loads still take
    // 4 wavefronts (rows of the piece 296 words, 8 banks, apart)
    const int lw = tid >> 5, ll = tid & 31;
    const int tx = (lw & 3) * 8 + (ll & 7), ty = (lw >> 2) * 4 + (ll >> 3);
    const int r = tr * kHvTile + ty, c = tc * kHvTile + tx;
    const bool valid = r < S.rows && c < S.cols;  // partial tiles at the far edges
    const long long p = valid ? (long long)r * S.cols + c : 0;
    const int own = (ty + kHvHalo) * kHvPitch + tx + kHvHalo;
    // the ground bit of the sweep's quads is the scene's (flags bit 0)
    const bool own_ground = valid && (statics ? (S.flags[p] & 1) != 0 : (bits[own] & 1u) != 0);
    const float ob = own_ground ? 1.f : 0.f;
    const uint32_t face = valid ? S.gvf_face[p] : 0u;
    constexpr float albedo_b = 0.2f;
    constexpr float inv_first = 1.f / FIRST, inv_first1 = 1.f / (FIRST + 1);
    constexpr float inv_second = 1.f / SECOND, inv_second1 = 1.f / (SECOND + 1);
    // walk lengths and the static plane: prepared with the scene
    // (gvf_statics_kernel) or walked here from the first daytime hour's quads
    uint32_t hits[4] = {0u, 0u, 0u, 0u};
    if (statics) {
        if (valid) {
#pragma unroll
            for (int w = 0; w < 4; ++w) hits[w] = S.gvf_hits[(long long)w * n + p];
            nosh[p] = S.gvf_nosh[p];
        }
    } else {
        const float nsh = hv_static_walks(bits, albs, own, own_ground, interior, r, c, S.rows, S.cols, tab, hits);
        if (valid) nosh[p] = nsh / 18.f;
    }
    const double ambient_e = valid ? kSBC * (double)S.emis[p] : 0.0;

    for (int g0 = 0; g0 < nd; g0 += kHvCh) {
        const int nc = nd - g0 < kHvCh ? nd - g0 : kHvCh;
        __syncthreads();  // the previous pass no longer reads the tile
        for (int i = tid; i < kHvN; i += kHvThreads) {
            const int rr = row0 + i / kHvPitch, cc = col0 + i % kHvPitch;
            const bool in = interior || in_raster(rr, cc, S.rows, S.cols);
            const long long pix = in ? (long long)rr * S.cols + cc : 0;
            float v[2 * kHvCh];
            uint32_t b = 0u;
#pragma unroll
            for (int k = 0; k < kHvCh; ++k) {
                if (k < nc && in) {
                    const float4 q = quads[(long long)dayh[g0 + k] * n + pix];
                    v[2 * k] = q.y;
                    v[2 * k + 1] = q.z * q.x;
                    b |= (((uint32_t)__float_as_int(q.w) & kQuadSunwall) ? 1u : 0u) << k;
                } else {
                    v[2 * k] = v[2 * k + 1] = 0.f;
                }
            }
            LA[i] = make_float4(v[0], v[1], v[2], v[3]);
            LB[i] = make_float4(v[4], v[5], v[6], v[7]);
            bits[i] = (uint8_t)b;
        }
        __syncthreads();
        float lw[kHvCh];
#pragma unroll
        for (int k = 0; k < kHvCh; ++k) {
            if (k < nc) {
                const SolweigHour& hh = hours[dayh[g0 + k]];
                lw[k] = (float)(kSBC * 0.9 * pow4(hh.tgwall + hh.ta + 273.15) - kSBC * 0.9 * pow4(hh.ta + 273.15));
            } else {
                lw[k] = 0.f;
            }
        }
        float lup_t[kHvCh], alb_t[kHvCh];
#pragma unroll
        for (int k = 0; k < kHvCh; ++k) lup_t[k] = alb_t[k] = 0.f;
        if (own_ground) {
#pragma unroll 1
            for (int j = 0; j < SOLWEIG_GVF_DIRECTIONS; ++j) {
                const uint32_t code = (hits[j / 5] >> (6 * (j % 5))) & 63u;
                const int lim = (int)(code & 31u);
                const int hit = (code & 32u) ? SECOND : lim;
                float sl[kHvCh], sa[kHvCh], l0[kHvCh], a0[kHvCh];
#pragma unroll
                for (int k = 0; k < kHvCh; ++k) sl[k] = sa[k] = l0[k] = a0[k] = 0.f;
                // Per hour k (byte k of both words): seen = a sunlit wall met so far,
                // cnt = steps before the first one (branch-free: each step adds
                // the not-yet-seen bytes), so f = cnt_k when seen_k.
                uint32_t seen = 0u, cnt = 0u;
#pragma unroll
                for (int m = 0; m < SECOND; ++m) {
                    if (m < lim) {
                        const int off = own + tab.delta[j * SECOND + m];
                        const float4 A = LA[off], B = LB[off];
                        const uint32_t b = bits[off];
                        sl[0] += A.x; sa[0] += A.y; sl[1] += A.z; sa[1] += A.w;
                        sl[2] += B.x; sa[2] += B.y; sl[3] += B.z; sa[3] += B.w;
                        seen |= (b * 0x00204081u) & 0x01010101u;  // bit k -> byte k
                        cnt += ~seen & 0x01010101u;
                        if (m + 1 == FIRST) {
#pragma unroll
                            for (int k = 0; k < kHvCh; ++k) {
                                l0[k] = sl[k];
                                a0[k] = sa[k];
                            }
                        }
                    }
                }
                if (hit > lim) {
                    // frozen tail (border tiles): step lim and the rest repeat step lim - 1,
                    // whose sunlit-wall bits are already counted
                    const int last = own + tab.delta[j * SECOND + lim - 1];
                    const float4 A = LA[last], B = LB[last];
                    const float rest = (float)(SECOND - 1 - lim);
                    const float tl[kHvCh] = {A.x, A.z, B.x, B.z}, ta_[kHvCh] = {A.y, A.w, B.y, B.w};
#pragma unroll
                    for (int k = 0; k < kHvCh; ++k) {
                        sl[k] += tl[k];
                        sa[k] += ta_[k];
                        sl[k] += rest * tl[k];
                        sa[k] += rest * ta_[k];
                    }
                }
                const bool fj = (face >> j) & 1u;
                // Per hour, with f the first step showing a sunlit wall (FIRST = 1):
                //   near = (f == 0 < hit): lup1 = (lw + l0) / 2, else l0;
                //   far  = (f < hit):      lup2 = ((SECOND - f) lw + sl) / (SECOND + 1), else sl / SECOND,
                //          the wall term dropped when f == 0 on a self-shadowed face (fj);
                //   lup_t += (0.5 lup1 + 0.4 lup2) / 0.9  (the same for the albedos with albedo_b),
                // as two fused multiply-adds with the selected weights.
#pragma unroll
                for (int k = 0; k < kHvCh; ++k) {
                    const int f = (seen >> (8 * k)) & 1u ? (int)((cnt >> (8 * k)) & 0xFFu) : 31;
                    const bool sun_far = f < hit;
                    const bool sun_near = sun_far && f == 0;
                    const float wn = (sun_far && !(sun_near && fj)) ? (float)(SECOND - f) : 0.f;
                    const float en = sun_near ? 1.f : 0.f;
                    const float c1 = sun_near ? (inv_first1 * 0.5f / 0.9f) : (inv_first * 0.5f / 0.9f);
                    const float c2 = sun_far ? (inv_second1 * 0.4f / 0.9f) : (inv_second * 0.4f / 0.9f);
                    lup_t[k] = fmaf(c1, fmaf(en, lw[k], l0[k]), lup_t[k]);
                    lup_t[k] = fmaf(c2, fmaf(wn, lw[k], sl[k]), lup_t[k]);
                    alb_t[k] = fmaf(c1, fmaf(en, albedo_b, a0[k]), alb_t[k]);
                    alb_t[k] = fmaf(c2, fmaf(wn, albedo_b, sa[k]), alb_t[k]);
                }
            }
        }
        const float4 oA = LA[own], oB = LB[own];
        const float own_lup[4] = {oA.x, oA.z, oB.x, oB.z};
        const float own_albsh[4] = {oA.y, oA.w, oB.y, oB.w};
#pragma unroll
        for (int k = 0; k < kHvCh; ++k) {
            if (k < nc && valid) {
                const int h = dayh[g0 + k];
                const SolweigHour& hh = hours[h];
                const float lt = lup_t[k] + 18.f * (own_lup[k] * (1.f - ob));
                const float at = alb_t[k] + 18.f * (own_albsh[k] * (1.f - ob));
                const double ambient = ambient_e * pow4(hh.ta + 273.15);
                gvf[(3LL * h) * n + p] = (float)((double)(lt / 18.f) + ambient);
                gvf[(3LL * h + 1) * n + p] = at / 18.f;
                gvf[(3LL * h + 2) * n + p] = quads[(long long)h * n + p].x;
            }
        }
    }
}

// Scene statics of the hour-vectorized GVF (1 m walk, no water): per pixel
// the walk-length codes [4][px] and the albedo-without-shadow GVF [px], from
// the scene's ground bits and albedo -- what day_gvf_hv_kernel would walk
// from the first daytime hour's quads each day.  32 x 32 tiles, 1024 threads.
size_t gvf_statics_smem_bytes() { return (size_t)kHvBitsBytes + (size_t)kHvN * sizeof(float); }

__global__ void __launch_bounds__(kHvThreads, 1) gvf_statics_kernel(SolweigScene S, GvfTable<22> tab,
                                                                   uint32_t* __restrict__ hits_out,
                                                                   float* __restrict__ nosh_out) {
    const int tr = blockIdx.y, tc = blockIdx.x;
    const bool interior = hv_tile_interior(S.rows, S.cols, tr, tc);
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float* albs = reinterpret_cast<float*>(smem_raw);
    uint8_t* bits = reinterpret_cast<uint8_t*>(albs + kHvN);
    const int tid = threadIdx.y * kHvTile + threadIdx.x;
    const long long n = (long long)S.rows * S.cols;
    const int row0 = tr * kHvTile - kHvHalo, col0 = tc * kHvTile - kHvHalo;
    for (int i = tid; i < kHvN; i += kHvThreads) {
        const int rr = row0 + i / kHvPitch, cc = col0 + i % kHvPitch;
        const bool in = interior || in_raster(rr, cc, S.rows, S.cols);
        const long long q = in ? (long long)rr * S.cols + cc : 0;
        bits[i] = in ? (uint8_t)(S.flags[q] & 1) : (uint8_t)0;
        albs[i] = in ? S.alb[q] : 0.f;
    }
    __syncthreads();
    const int lw = tid >> 5, ll = tid & 31;
    const int tx = (lw & 3) * 8 + (ll & 7), ty = (lw >> 2) * 4 + (ll >> 3);
    const int r = tr * kHvTile + ty, c = tc * kHvTile + tx;
    if (r >= S.rows || c >= S.cols) return;
    const long long p = (long long)r * S.cols + c;
    const int own = (ty + kHvHalo) * kHvPitch + tx + kHvHalo;
    const bool own_ground = (bits[own] & 1u) != 0;
    uint32_t hits[4];
    const float nsh = hv_static_walks(bits, albs, own, own_ground, interior, r, c, S.rows, S.cols, tab, hits);
#pragma unroll
    for (int w = 0; w < 4; ++w) hits_out[(long long)w * n + p] = hits[w];
    nosh_out[p] = nsh / 18.f;
}

// ------------------------------------------------------------- kernels 3, 4, 5

// w[2h][k] = luminance, w[2h+1][k] = luminance * cos(alt) * omega (0 at night).
__global__ void day_weights_kernel(const SolweigSkyLayout* __restrict__ L, const SolweigHour* __restrict__ hours,
                                   int nhours, float* __restrict__ w) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= 2 * nhours * kK) return;
    const int row = idx / kK, k = idx - row * kK;
    const SolweigHour& h = hours[row >> 1];
    float v = 0.f;
    if (h.daytime && k < L->patches) v = (row & 1) ? h.lum[k] * L->cos_alt[k] * L->omega[k] : h.lum[k];
    w[idx] = v;
}

// BF16 hi/lo split of scale * w [ncols][kK] into the canonical operand layout
// b[0][nb rows] (hi) and b[1][nb rows] (lo); rows >= ncols are zero.
__global__ void split_bf16_kernel(const float* __restrict__ w, int ncols, int nb, int patches,
                                  __nv_bfloat16* __restrict__ b, float scale = 1.f) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= nb * kK) return;
    const int n = idx / kK, k = idx - n * kK;
    const float v = (n < ncols && k < patches) ? scale * w[n * kK + k] : 0.f;
    const __nv_bfloat16 hi = __float2bfloat16_rn(v);
    const __nv_bfloat16 lo = __float2bfloat16_rn(v - __bfloat162float(hi));
    const int o = canon_off(n, k);
    b[o] = hi;
    b[nb * kK + o] = lo;
}

// One block per hour, kK threads.
__global__ void __launch_bounds__(kK) day_tables_kernel(const SolweigSkyLayout* __restrict__ L,
                                                        const SolweigHour* __restrict__ hours,
                                                        DayTable* __restrict__ tables) {
    __shared__ double ts[kK], vs[kK];
    __shared__ int perm_t[kK], perm_v[kK];
    const SolweigHour& h = hours[blockIdx.x];
    DayTable& T = tables[blockIdx.x];
    const int P = L->patches;
    const int k = threadIdx.x;
    double tk = 0.0, vk = 0.0;
    if (k < P) {
        const double yi = h.yi[k], lo = L->sunlit_below[k], hi = L->shaded_above[k];
        tk = first_true([&](double t) { return !((t + yi) < lo); });
        vk = first_true([&](double t) { return (t + yi) > hi; });
        ts[k] = tk;
        vs[k] = vk;
    }
    __syncthreads();
    if (k < P) {
        int rt = 0, rv = 0;
        for (int j = 0; j < P; ++j) {
            rt += (ts[j] < tk || (ts[j] == tk && j < k)) ? 1 : 0;
            rv += (vs[j] < vk || (vs[j] == vk && j < k)) ? 1 : 0;
        }
        T.tsun[rt] = tk;
        T.vshade[rv] = vk;
        perm_t[rt] = k;
        perm_v[rv] = k;
    }
    __syncthreads();
    for (int i = k; i <= P; i += blockDim.x) {
        uint32_t suf[SOLWEIG_MASK_WORDS] = {0, 0, 0, 0, 0}, pre[SOLWEIG_MASK_WORDS] = {0, 0, 0, 0, 0};
        for (int r = 0; r < P; ++r) {
            if (r >= i) suf[perm_t[r] >> 5] |= 1u << (perm_t[r] & 31);
            if (r < i) pre[perm_v[r] >> 5] |= 1u << (perm_v[r] & 31);
        }
        for (int w = 0; w < SOLWEIG_MASK_WORDS; ++w) {
            T.suf[i][w] = suf[w];
            T.pre[i][w] = pre[w];
        }
    }
    if (k < SOLWEIG_MASK_WORDS) {
        uint32_t t = 0;
        for (int b = 0; b < 32; ++b) {
            const int kk = k * 32 + b;
            if (kk < P && h.daytime && h.lw_sun_test[kk]) t |= 1u << b;
        }
        T.test[k] = t;
    }
    __syncthreads();  // sorted arrays complete
    for (int i = k; i < 256; i += blockDim.x) {
        const double bound = tan_bucket_bound(i);
        int ns = 0, nv = 0;
        for (int j = 0; j < P; ++j) {
            ns += T.tsun[j] < bound ? 1 : 0;
            nv += T.vshade[j] < bound ? 1 : 0;
        }
        T.sun_start[i] = (uint8_t)ns;
        T.shd_start[i] = (uint8_t)nv;
    }
    if (k < SOLWEIG_MAX_BANDS) {
        const bool ok = k < L->nbands;
        T.band_down[k] = ok ? h.band_lsky[k] * L->band_omega[k] * L->band_sin[k] : 0.f;
        T.band_side[k] = ok ? h.band_lsky[k] * L->band_omega[k] * L->band_cos[k] : 0.f;
    }
    if (k == 32) {
        const double tk = h.ta + 273.15;
        T.lw_shade = (float)((0.9 * kSBC * pow4(tk)) / kPi);
        T.lw_sun = h.daytime ? (float)((0.9 * kSBC * pow4(h.ta + h.tgwall + 273.15)) / kPi) : 0.f;
        T.sw_shade = (float)((0.2 * h.rad_d * 0.5) / kPi);
        T.sw_sun = (float)((0.2 * (h.rad_i * h.cos_alt) + h.rad_d * 0.5) / kPi);
        T.rad_d = (float)h.rad_d;
        T.rad_g = (float)h.rad_g;
        T.direct_up = (float)(h.rad_i * h.sin_alt);
        T.rad_i_sin = (float)(h.rad_i * h.sin_alt);
        T.rad_i_cos = (float)(h.rad_i * h.cos_alt);
        T.rad_ratio = (float)(h.rad_d / h.rad_tot);
        T.wave_w = (float)h.wave_weight;
        T.tan_zen = (float)h.tan_zen;
        T.night_lup = (float)(kSBC * pow4(tk));
        T.night_lup_water = (float)(kSBC * 0.98 * pow4(h.twater + 273.15));
    }
}

// ------------------------------------------------------------------ kernel 6

struct GemmArgs {
    const uint32_t* masks;  // S/V bit planes [10][px]
    long long px;
    int patches;
    const __nv_bfloat16* b;  // [2][nb * kK] canonical hi, lo (combined: [4][nb * kK], then c * w hi, lo)
    int ncols, nb;
    float* out;  // [2 * ncols][px]: sky columns, then vegetation columns (combined: [ncols][px])
    int* error;
    // 1: one set of columns, sky sums plus the vegetation sums of weights
    // prescaled by c (the diffuse transmissivity of vegetation): both MMA
    // pairs accumulate into the same tensor-memory columns
    int combined;
};

size_t gemm_smem_bytes(int nb, bool combined) {
    return (size_t)2 * kABytes + (size_t)(combined ? 4 : 2) * nb * kK * 2 + 16;
}

// Expand 8 mask bits to 8 BF16 values (1.0 or 0.0) packed in a uint4.
// t = byte + (byte << 15) holds bit 2i at position 2i and bit 2i + 1 at
// position 16 + 2i, so (t >> 2i) & 0x10001 has the pair's two bits at 0 and
// 16, and times 0x3F80 (BF16 1.0) gives the two packed values.
__device__ __forceinline__ uint4 expand8(uint32_t byte) {
    const uint32_t t = byte * 0x8001u;
    uint32_t v[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) v[i] = ((t >> (2 * i)) & 0x10001u) * 0x3F80u;
    return make_uint4(v[0], v[1], v[2], v[3]);
}

// Persistent: one 128-pixel tile per iteration.  All 128 threads expand the
// tile's masks into the two A operands; thread 0 issues the MMAs (sky and
// vegetation, BF16 hi and lo weights accumulating into the same FP32
// columns) and commits them to an mbarrier; each warp then reads its 32 rows
// (pixels) of the accumulators from tensor memory and stores them.
__global__ void __launch_bounds__(kARows, 1) patch_gemm_kernel(GemmArgs g) {
    extern __shared__ __align__(1024) unsigned char smem[];
    unsigned char* a_sky = smem;
    unsigned char* a_veg = smem + kABytes;
    unsigned char* b_ops = smem + 2 * kABytes;  // hi then lo (combined: then c * w hi, lo)
    const int bbytes = g.nb * kK * 2;
    const int nbops = g.combined ? 4 : 2;
    uint64_t* bar = reinterpret_cast<uint64_t*>(b_ops + nbops * bbytes);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bar + 1);
    const int tid = threadIdx.x, warp = tid >> 5;
    uint32_t ncols_tmem = 32;
    while (ncols_tmem < (uint32_t)((g.combined ? 1 : 2) * g.nb)) ncols_tmem <<= 1;

    {  // weights: global -> shared, 16 bytes per copy
        const uint4* src = reinterpret_cast<const uint4*>(g.b);
        uint4* dst = reinterpret_cast<uint4*>(b_ops);
        for (int i = tid; i < nbops * bbytes / 16; i += blockDim.x) dst[i] = src[i];
    }
    if (tid == 0) {
        tc::mbar_init(bar, 1);
        tc::fence_mbar_init();
    }
    if (warp == 0) {
        tc::tmem_alloc(tmem_slot, ncols_tmem);
        tc::tmem_relinquish();
    }
    tc::fence_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *tmem_slot;
    const uint32_t idesc = tc::idesc_bf16_f32(kARows, g.nb);
    const uint32_t a_sky_addr = tc::smem_addr(a_sky), a_veg_addr = tc::smem_addr(a_veg);
    const uint32_t b_hi_addr = tc::smem_addr(b_ops), b_lo_addr = b_hi_addr + bbytes;
    uint32_t valid[SOLWEIG_MASK_WORDS];
#pragma unroll
    for (int w = 0; w < SOLWEIG_MASK_WORDS; ++w) {
        const int nbits = g.patches - 32 * w;
        valid[w] = nbits >= 32 ? 0xffffffffu : (nbits <= 0 ? 0u : ((1u << nbits) - 1u));
    }
    const long long ntiles = (g.px + kARows - 1) / kARows;
    uint32_t phase = 0;
    bool failed = false;
    for (long long t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const long long p = t * kARows + tid;
        const bool in = p < g.px;
        // Expand this pixel's row of both A operands.
        unsigned char* row_sky = a_sky + (tid >> 3) * kSBO + (tid & 7) * 16;
        unsigned char* row_veg = a_veg + (tid >> 3) * kSBO + (tid & 7) * 16;
#pragma unroll
        for (int w = 0; w < SOLWEIG_MASK_WORDS; ++w) {
            const uint32_t s = in ? g.masks[(long long)w * g.px + p] : 0u;
            const uint32_t v = in ? g.masks[(long long)(SOLWEIG_MASK_WORDS + w) * g.px + p] : 0u;
            const uint32_t sky = s & ~v & valid[w], veg = s & v & valid[w];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int chunk = w * 4 + j;
                *reinterpret_cast<uint4*>(row_sky + chunk * 128) = expand8((sky >> (8 * j)) & 0xFFu);
                *reinterpret_cast<uint4*>(row_veg + chunk * 128) = expand8((veg >> (8 * j)) & 0xFFu);
            }
        }
        tc::fence_async_smem();
        __syncthreads();
        if (tid == 0) {
            tc::fence_after_sync();
#pragma unroll 1
            for (int s = 0; s < kK / 16; ++s) {
                const uint64_t bh = tc::smem_desc(b_hi_addr + s * 256, 128, kSBO);
                const uint64_t bl = tc::smem_desc(b_lo_addr + s * 256, 128, kSBO);
                const uint64_t as = tc::smem_desc(a_sky_addr + s * 256, 128, kSBO);
                const uint64_t av = tc::smem_desc(a_veg_addr + s * 256, 128, kSBO);
                tc::mma_bf16(tmem, as, bh, idesc, s > 0);
                tc::mma_bf16(tmem, as, bl, idesc, true);
                if (g.combined) {
                    const uint64_t ch = tc::smem_desc(b_hi_addr + 2 * bbytes + s * 256, 128, kSBO);
                    const uint64_t cl = tc::smem_desc(b_hi_addr + 3 * bbytes + s * 256, 128, kSBO);
                    tc::mma_bf16(tmem, av, ch, idesc, true);
                    tc::mma_bf16(tmem, av, cl, idesc, true);
                } else {
                    tc::mma_bf16(tmem + g.nb, av, bh, idesc, s > 0);
                    tc::mma_bf16(tmem + g.nb, av, bl, idesc, true);
                }
            }
            tc::mma_commit(bar);
        }
        const bool ok = tc::mbar_wait(bar, phase, kWaitPolls);
        if (__syncthreads_or(!ok)) {
            failed = true;
            break;
        }
        phase ^= 1u;
        tc::fence_after_sync();
        const uint32_t lane_base = tmem + ((uint32_t)(warp * 32) << 16);
        if (g.combined) {
            for (int c0 = 0; c0 < g.ncols; c0 += 8) {
                float vs[8];
                tc::tmem_ld8(lane_base + c0, vs);
                tc::tmem_wait_ld();
                if (in) {
#pragma unroll
                    for (int i = 0; i < 8; ++i)
                        if (c0 + i < g.ncols) g.out[(long long)(c0 + i) * g.px + p] = vs[i];
                }
            }
        } else {
            for (int c0 = 0; c0 < g.ncols; c0 += 8) {
                float vs[8], vv[8];
                tc::tmem_ld8(lane_base + c0, vs);
                tc::tmem_ld8(lane_base + g.nb + c0, vv);
                tc::tmem_wait_ld();
                if (in) {
#pragma unroll
                    for (int i = 0; i < 8; ++i) {
                        if (c0 + i < g.ncols) {
                            g.out[(long long)(c0 + i) * g.px + p] = vs[i];
                            g.out[(long long)(g.ncols + c0 + i) * g.px + p] = vv[i];
                        }
                    }
                }
            }
        }
        tc::fence_before_sync();
        __syncthreads();
    }
    if (failed) {
        if (tid == 0) raise_day_flag(g.error, 1);
        // let the MMAs of the abandoned tile finish before freeing their columns
        tc::mbar_wait(bar, phase, kWaitPolls);
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        tc::fence_after_sync();
        tc::tmem_dealloc(tmem, ncols_tmem);
    }
}

// Pipelined form of the combined contraction (the batched day's): two A
// stages in shared memory and two accumulators in tensor memory, 256
// threads.  While the tensor cores multiply tile i, the threads expand tile
// i + 1 into the other stage (threads 0-127 the sky masks, 128-255 the
// vegetation masks of the same 128 pixels; the mask words of tile i + 2 are
// already loading), then wait for tile i and store its sums from tensor
// memory (warp w: lanes 32 (w % 4) .. + 31, every other 8-column group from
// 8 (w / 4)).  Thread 0 issues each tile's MMAs once both of its operands
// are in shared memory and the stage's accumulator has been read out.
constexpr int kPipeThreads = 2 * kARows;

size_t gemm_pipe_smem_bytes(int nb) { return (size_t)4 * kABytes + (size_t)4 * nb * kK * 2 + 32; }

__global__ void __launch_bounds__(kPipeThreads, 1) patch_gemm_pipe_kernel(GemmArgs g) {
    extern __shared__ __align__(1024) unsigned char smem[];
    unsigned char* b_ops = smem + 4 * kABytes;  // hi, lo, c * w hi, c * w lo
    const int bbytes = g.nb * kK * 2;
    uint64_t* bar = reinterpret_cast<uint64_t*>(b_ops + 4 * bbytes);  // one per stage
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bar + 2);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int row = tid & (kARows - 1);
    const bool veg_half = tid >= kARows;
    uint32_t ncols_tmem = 32;
    while (ncols_tmem < (uint32_t)(2 * g.nb)) ncols_tmem <<= 1;
    {  // weights: global -> shared, 16 bytes per copy
        const uint4* src = reinterpret_cast<const uint4*>(g.b);
        uint4* dst = reinterpret_cast<uint4*>(b_ops);
        for (int i = tid; i < 4 * bbytes / 16; i += blockDim.x) dst[i] = src[i];
    }
    if (tid == 0) {
        tc::mbar_init(&bar[0], 1);
        tc::mbar_init(&bar[1], 1);
        tc::fence_mbar_init();
    }
    if (warp == 0) {
        tc::tmem_alloc(tmem_slot, ncols_tmem);
        tc::tmem_relinquish();
    }
    tc::fence_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *tmem_slot;
    const uint32_t idesc = tc::idesc_bf16_f32(kARows, g.nb);
    const uint32_t b_hi_addr = tc::smem_addr(b_ops);
    uint32_t valid[SOLWEIG_MASK_WORDS];
#pragma unroll
    for (int w = 0; w < SOLWEIG_MASK_WORDS; ++w) {
        const int nbits = g.patches - 32 * w;
        valid[w] = nbits >= 32 ? 0xffffffffu : (nbits <= 0 ? 0u : ((1u << nbits) - 1u));
    }
    const long long ntiles = (g.px + kARows - 1) / kARows;
    const long long first = blockIdx.x, stride = gridDim.x;
    const long long my = first < ntiles ? (ntiles - 1 - first) / stride + 1 : 0;  // tiles of this CTA

    uint32_t sw[SOLWEIG_MASK_WORDS], vw[SOLWEIG_MASK_WORDS];
    auto load = [&](long long t) {
        const long long p = t * kARows + row;
        const bool in = p < g.px;
#pragma unroll
        for (int w = 0; w < SOLWEIG_MASK_WORDS; ++w) {
            sw[w] = in ? __ldg(&g.masks[(long long)w * g.px + p]) : 0u;
            vw[w] = in ? __ldg(&g.masks[(long long)(SOLWEIG_MASK_WORDS + w) * g.px + p]) : 0u;
        }
    };
    auto expand = [&](int st) {
        unsigned char* a = smem + (2 * st + (veg_half ? 1 : 0)) * kABytes;
        unsigned char* rowp = a + (row >> 3) * kSBO + (row & 7) * 16;
#pragma unroll
        for (int w = 0; w < SOLWEIG_MASK_WORDS; ++w) {
            const uint32_t m = (veg_half ? (sw[w] & vw[w]) : (sw[w] & ~vw[w])) & valid[w];
#pragma unroll
            for (int j = 0; j < 4; ++j)
                *reinterpret_cast<uint4*>(rowp + (w * 4 + j) * 128) = expand8((m >> (8 * j)) & 0xFFu);
        }
    };
    auto issue = [&](int st) {  // thread 0: sky x (hi, lo) and vegetation x (c hi, c lo) into stage st
        tc::fence_after_sync();
        const uint32_t acc = tmem + (uint32_t)(st * g.nb);
        const uint32_t as0 = tc::smem_addr(smem + 2 * st * kABytes), av0 = as0 + kABytes;
#pragma unroll 1
        for (int k = 0; k < kK / 16; ++k) {
            const uint64_t bh = tc::smem_desc(b_hi_addr + k * 256, 128, kSBO);
            const uint64_t bl = tc::smem_desc(b_hi_addr + bbytes + k * 256, 128, kSBO);
            const uint64_t ch = tc::smem_desc(b_hi_addr + 2 * bbytes + k * 256, 128, kSBO);
            const uint64_t cl = tc::smem_desc(b_hi_addr + 3 * bbytes + k * 256, 128, kSBO);
            const uint64_t as = tc::smem_desc(as0 + k * 256, 128, kSBO);
            const uint64_t av = tc::smem_desc(av0 + k * 256, 128, kSBO);
            tc::mma_bf16(acc, as, bh, idesc, k > 0);
            tc::mma_bf16(acc, as, bl, idesc, true);
            tc::mma_bf16(acc, av, ch, idesc, true);
            tc::mma_bf16(acc, av, cl, idesc, true);
        }
        tc::mma_commit(&bar[st]);
    };

    uint32_t parity[2] = {0u, 0u};
    int pending = 0;  // stages with committed MMAs not yet waited for
    bool failed = false;
    if (my > 0) {
        load(first);
        expand(0);
        if (my > 1) load(first + stride);
        tc::fence_async_smem();
        __syncthreads();
        if (tid == 0) issue(0);
        pending = 1;
    }
    for (long long i = 0; i < my; ++i) {
        const int st = (int)(i & 1);
        const long long t = first + i * stride;
        if (i + 1 < my) {
            expand(st ^ 1);  // its masks were loaded one iteration ago
            if (i + 2 < my) load(t + 2 * stride);
        }
        tc::fence_async_smem();
        tc::fence_before_sync();
        __syncthreads();  // stage st ^ 1 expanded; its accumulator read out last iteration
        if (i + 1 < my) {
            if (tid == 0) issue(st ^ 1);
            pending |= 1 << (st ^ 1);
        }
        const bool ok = tc::mbar_wait(&bar[st], parity[st], kWaitPolls);
        if (__syncthreads_or(!ok)) {
            failed = true;
            break;
        }
        parity[st] ^= 1u;
        pending &= ~(1 << st);
        tc::fence_after_sync();
        const int q = warp & 3;
        const uint32_t lane_base = tmem + (uint32_t)(st * g.nb) + ((uint32_t)(q * 32) << 16);
        const long long p = t * kARows + q * 32 + lane;
        const bool in = p < g.px;
        for (int c0 = 8 * (warp >> 2); c0 < g.ncols; c0 += 16) {
            float v[8];
            tc::tmem_ld8(lane_base + c0, v);
            tc::tmem_wait_ld();
            if (in) {
#pragma unroll
                for (int k = 0; k < 8; ++k)
                    if (c0 + k < g.ncols) g.out[(long long)(c0 + k) * g.px + p] = v[k];
            }
        }
    }
    if (failed) {
        if (tid == 0) raise_day_flag(g.error, 1);
        // let committed MMAs finish before their columns are freed
        for (int st = 0; st < 2; ++st)
            if (pending & (1 << st)) tc::mbar_wait(&bar[st], parity[st], kWaitPolls);
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        tc::fence_after_sync();
        tc::tmem_dealloc(tmem, ncols_tmem);
    }
}

// ------------------------------------------------------------------ kernel 7

struct DayRadArgs {
    const SolweigSkyLayout* layout;
    const SolweigHour* hours;
    int nhours;
    const DayTable* tables;
    const float* gvf;   // [H][3][px]
    const float* nosh;  // [px]
    const float* sums;  // [ncols][px]: sky + 0.03 x vegetation sums (luminance, luminance*cos*omega)
    int ncols;
    SolweigState state;
    SolweigOutputs out;  // base pointers; hour h at + h * hour_stride
    long long hour_stride;
};


__device__ __forceinline__ float* hour_plane(float* base, int hr, long long stride) {
    return base ? base + hr * stride : nullptr;
}

// Fraction of shaded wall (cylindric_wedge, NaN -> 0.5) in float32.
__device__ __forceinline__ float wedge_fsh_f(float ta, float tan_zen) {
    const float xa = 1.f - 2.f / (ta * tan_zen);
    const float ha = 2.f / (ta * tan_zen);
    const float ba = 1.f / ta;
    const float hkil = 2.f * ba * ha;
    float ukil = 0.f;
    if (xa < 0.f) {
        // phi = atan(za / qa) in [0, pi/2): cos and sin from the same triangle,
        // 1 / hypot(qa, za) with qa^2 + za^2 = ba^2 + 3 qa^2 / 4
        const float qa = tan_zen / 2.f;
        const float za = sqrtf(ba * ba - qa * qa / 4.f);
        const float phi = atanf(za / qa);
        const float ih = rsqrtf(fmaf(qa, qa, za * za));
        const float cphi = qa * ih, sphi = za * ih;
        const float area = (sphi - phi * cphi) / (1.f - cphi);
        ukil = 2.f * ba * xa * area;
    }
    const float pi2 = 2.f * (float)kPi;
    const float fsh = (pi2 * ba - (hkil + ukil)) / (pi2 * ba);
    return isnan(fsh) ? 0.5f : fsh;
}

// Flux arithmetic of the hour loop in float32 (the hour's scalars are
// staged once per block, rounded from the float64 host plan); the building
// split keeps its exact float64 thresholds.  Against the per-hour form
// (float64 fluxes) Tmrt differs by < 1e-3 K (tested).  Launched for full
// occupancy, 2048 resident threads per SM (32 registers): the loop is
// latency-bound, and the extra warps outweigh the spilled registers (per
// 2000^2 day: 5.65 ms at 512 threads, 4.32 at 768, 3.70 at 1024, 3.46 at
// 1280, 3.26 at 1536, 3.15 at 2048).  The hour tables and scalars are read
// from the day's table array through L1 instead of being staged in shared
// memory, so the hour loop has no barrier (3.15 -> 2.92 ms).
template <int OPT, int THREADS>
__global__ void __launch_bounds__(THREADS, 2048 / THREADS) day_radiation_kernel(SolweigScene S, DayRadArgs a) {
    __shared__ float wcos[SOLWEIG_MAX_BANDS], wsin[SOLWEIG_MAX_BANDS];
    const SolweigSkyLayout& L = *a.layout;
    if (threadIdx.x < SOLWEIG_MAX_BANDS) {
        const int b = threadIdx.x;
        const int k0 = Bands<OPT>::off(b < 8 ? b : 0);
        wcos[b] = b < L.nbands ? L.omega[k0] * L.cos_alt[k0] : 0.f;
        wsin[b] = b < L.nbands ? L.omega[k0] * L.sin_alt[k0] : 0.f;
    }
    __syncthreads();  // wcos, wsin
    const long long n = (long long)S.rows * S.cols;
    const long long p = (long long)blockIdx.x * THREADS + threadIdx.x;
    const bool in = p < n;
    const long long q = in ? p : 0;  // a valid pixel for the loads of idle threads
    const SolweigOutputs& o = a.out;
    const bool need_tg = o.tg || o.tg_out || a.state.tgout1;

    // --- per-pixel static data, loaded once for the day
    uint32_t bld[SOLWEIG_MASK_WORDS];
#pragma unroll
    for (int w = 0; w < SOLWEIG_MASK_WORDS; ++w) {
        const int nbits = S.patches - 32 * w;
        const uint32_t valid = nbits >= 32 ? 0xffffffffu : (nbits <= 0 ? 0u : ((1u << nbits) - 1u));
        bld[w] = ~S.masks[(long long)w * n + q] & ~S.masks[(long long)(SOLWEIG_MASK_WORDS + w) * n + q] & valid;
    }
    uint32_t cnt_lo = 0, cnt_hi = 0;  // sky patches per band, 8 bits each
#pragma unroll
    for (int b = 0; b < 4; ++b) {
        cnt_lo |= (uint32_t)S.sky_band_counts[(long long)b * n + q] << (8 * b);
        cnt_hi |= (uint32_t)(b + 4 < S.nbands ? S.sky_band_counts[(long long)(b + 4) * n + q] : 0) << (8 * b);
    }
    const uint8_t fl = S.flags[q];
    const bool ground = fl & 1;
    const bool water = S.has_water && (fl & 4);
    const float emis = S.emis[q];
    const float svfbuveg = S.svfbuveg[q];
    const float tan_alfa = (float)tan(S.svfalfa[q]);
    const double tan_asvf = S.tan_asvf[q];
    const int tbucket = tan_bucket(tan_asvf);
    const float vc = S.veg_sums[q], vs = S.veg_sums[n + q];
    const float oc = S.veg_sums[2 * n + q], os = S.veg_sums[3 * n + q];
    const float g_nosh = a.nosh[q];
    constexpr float ewall = 0.9f, albedo_b = 0.2f;
    constexpr float absK = 0.7f, absL = 0.95f, Fside = 0.22f, Fup = 0.06f, Fcyl = 0.28f;
    constexpr float dsh_veg = 0.03f;
    constexpr float sbc = (float)kSBC, inv_pi = (float)(1.0 / kPi);

    float st_lup = a.state.tgmap1 ? a.state.tgmap1[q] : 0.f;
    float st_tg = a.state.tgout1 ? a.state.tgout1[q] : 0.f;

    for (int hr = 0; hr < a.nhours; ++hr) {
        // the hour's table and scalars, read through L1 by every thread (no
        // shared staging, so the hour loop needs no barrier)
        const DayTable& hs = a.tables[hr];
        const SolweigHour& h = a.hours[hr];
        const bool day = h.daytime != 0;
        const float ta = (float)h.ta;

        // building patches: sunlit / shaded split of the hour
        const DayTable& T = hs;
        const int P = S.patches;
        const int isun = count_le_from(T.tsun, P, T.sun_start[tbucket], tan_asvf);
        const int ishd = count_le_from(T.vshade, P, T.shd_start[tbucket], tan_asvf);
        uint32_t m_sun[SOLWEIG_MASK_WORDS], m_shd[SOLWEIG_MASK_WORDS], m_lsun[SOLWEIG_MASK_WORDS],
            m_lshd[SOLWEIG_MASK_WORDS];
#pragma unroll
        for (int w = 0; w < SOLWEIG_MASK_WORDS; ++w) {
            const uint32_t test = T.test[w];
            m_sun[w] = bld[w] & T.suf[isun][w];
            m_shd[w] = bld[w] & T.pre[ishd][w];
            m_lsun[w] = m_sun[w] & test;
            m_lshd[w] = bld[w] & (~test | m_shd[w]);
        }
        float cnt_lsun[8], cnt_lshd[8];
        band_counts<OPT>(m_lsun, cnt_lsun);
        band_counts<OPT>(m_lshd, cnt_lshd);
        const float lw_sun_c = band_dot(cnt_lsun, wcos), lw_sun_s = band_dot(cnt_lsun, wsin);
        const float lw_shd_c = band_dot(cnt_lshd, wcos), lw_shd_s = band_dot(cnt_lshd, wsin);
        float ld_sky = 0.f, ls_sky = 0.f;
#pragma unroll
        for (int b = 0; b < 8; ++b) {
            const float cnt = (float)(((b < 4 ? cnt_lo : cnt_hi) >> (8 * (b & 3))) & 0xFFu);
            ld_sky = fmaf(hs.band_down[b], cnt, ld_sky);
            ls_sky = fmaf(hs.band_side[b], cnt, ls_sky);
        }
        const float lw_shade = hs.lw_shade, lw_sun = hs.lw_sun;

        float shadow = 0.f, tg = 0.f, tg_out = ta;
        float kup_all = 0.f, lup_all;
        float kdown = 0.f, kside = 0.f, kside_i = 0.f, kside_d = 0.f, d_rad = 0.f;
        if (day) {
            const long long g0 = (3LL * hr) * n + q;
            const float g_lup = a.gvf[g0];
            const float g_alb = a.gvf[g0 + n];
            shadow = a.gvf[g0 + 2 * n];
            const float fsh = wedge_fsh_f(tan_alfa, hs.tan_zen);
            const float reflected = albedo_b * (1.f - svfbuveg) * (hs.rad_g * (1.f - fsh) + hs.rad_d * fsh);
            const float base_up = hs.rad_d * svfbuveg + reflected;
            kup_all = g_alb * hs.direct_up + base_up * g_nosh;
            const float prev = h.firstdaytime ? g_lup : st_lup;
            lup_all = g_lup * (1.f - hs.wave_w) + prev * hs.wave_w;
            st_lup = h.wave_update ? lup_all : prev;
            if (need_tg) {
                // ground temperature (TsWaveDelay of Tg * shadow + Ta); not part of Tmrt
                const double amp = (double)S.tgk[q] * h.altmax + (double)S.tstart[q];
                const double phase = ((h.dectime_frac - h.snup / 24.0) /
                                      ((double)S.tmaxlst[q] / 24.0 - h.snup / 24.0)) * kPi / 2.0;
                double tgd = amp * sin(phase) * h.ci_tgg;
                if (S.landcover == 1 && tgd < 0.0) tgd = 0.0;
                if (water) tgd = h.twater - h.ta;
                tg = (float)tgd;
                const float cur = tg * shadow + ta;
                const float prv = h.firstdaytime ? cur : st_tg;
                tg_out = cur * (1.f - hs.wave_w) + prv * hs.wave_w;
                st_tg = h.wave_update ? tg_out : prv;
            }
            // the contraction already added the vegetation patches at their
            // diffuse transmissivity (dsh_veg): sky + dsh_veg x vegetation sums
            const long long s0 = 2LL * hr;
            const float lum = a.sums[s0 * n + q], cw = a.sums[(s0 + 1) * n + q];
            d_rad = hs.rad_d * lum;
            kdown = hs.rad_i_sin * shadow + d_rad + reflected;
            kside_i = shadow * hs.rad_i_cos;
            kside_d = hs.rad_ratio * cw;
            kside = kside_i + kside_d + hs.sw_sun * band_weighted<OPT>(m_sun, wcos) +
                    hs.sw_shade * band_weighted<OPT>(m_shd, wcos) + hs.sw_shade * vc;
        } else {
            float lup = emis * hs.night_lup;
            if (S.landcover == 1 && (fl & 4)) lup = hs.night_lup_water;
            lup_all = lup;
        }
        const float refl = (ld_sky + lup_all) * ((1.f - ewall) * 0.5f * inv_pi);
        const float ldown = ld_sky + lw_shade * vs + lw_shade * lw_shd_s + lw_sun * lw_sun_s + refl * os;
        const float lside = ls_sky + lw_shade * vc + lw_shade * lw_shd_c + lw_sun * lw_sun_c + refl * oc;
        // E+S+W+N of Kup and Lup are 4x the all-direction values (see the file header).
        const float sstr = absK * (kside * Fcyl + (kdown + kup_all) * Fup + 2.f * kup_all * Fside) +
                           absL * ((ldown + lup_all) * Fup + lside * Fcyl + 2.f * lup_all * Fside);
        const float tmrt = sqrtf(sqrtf(sstr * (1.f / (absL * sbc)))) - 273.2f;
        if (in) {
            const long long hs_ = a.hour_stride;
            if (o.tmrt) o.tmrt[hr * hs_ + p] = tmrt;
            if (o.utci)
                o.utci[hr * hs_ + p] = ground ? utci_eval(h.utci, (double)tmrt, h.ta, h.utci_valid)
                                              : __int_as_float(0x7fc00000);
            if (o.kdown) o.kdown[hr * hs_ + p] = kdown;
            if (o.kup) o.kup[hr * hs_ + p] = kup_all;
            if (o.ldown) o.ldown[hr * hs_ + p] = ldown;
            if (o.lup) o.lup[hr * hs_ + p] = lup_all;
            if (o.lside) o.lside[hr * hs_ + p] = lside;
            if (o.kside_i) o.kside_i[hr * hs_ + p] = kside_i;
            if (o.kside_d) o.kside_d[hr * hs_ + p] = kside_d;
            if (o.kside) o.kside[hr * hs_ + p] = kside;
            if (o.d_rad) o.d_rad[hr * hs_ + p] = d_rad;
            if (o.shadow) o.shadow[hr * hs_ + p] = shadow;
            if (o.tg) o.tg[hr * hs_ + p] = tg;
            if (o.tg_out) o.tg_out[hr * hs_ + p] = tg_out;
        }
    }
    if (in) {
        if (a.state.tgmap1) a.state.tgmap1[p] = st_lup;
        if (a.state.tgout1) a.state.tgout1[p] = st_tg;
    }
}

// ------------------------------------------------------------------ host side

inline long long align256(long long x) { return (x + 255) & ~255LL; }

struct DayWork {
    long long quads, lup_first, gvf, nosh, sums, wf32, bw, tables, error, tilemax, total;
};

DayWork day_work_layout(long long px, int nhours, bool water) {
    DayWork w{};
    const int ncols = 2 * nhours;
    const int nb = (ncols + 15) / 16 * 16;
    long long o = 0;
    // the error flag pair first: the same place for every raster size, so the
    // days of differently sized tiles sharing one buffer share its sticky word
    w.error = o; o = align256(o + 16);
    w.quads = o; o = align256(o + 16LL * px * nhours);
    w.lup_first = o; o = align256(o + (water ? 4LL * px * nhours : 0));
    w.gvf = o; o = align256(o + 12LL * px * nhours);
    w.nosh = o; o = align256(o + 4LL * px);
    w.sums = o; o = align256(o + 4LL * px * 2 * ncols);
    w.wf32 = o; o = align256(o + 4LL * ncols * kK);
    w.bw = o; o = align256(o + 2LL * 4 * nb * kK);
    w.tables = o; o = align256(o + (long long)sizeof(DayTable) * nhours);
    // per 16 x 16 tile maxima of the heights (ceil(rows/16) * ceil(cols/16)
    // floats, bounded here from the pixel count alone: <= px/256 + (rows + cols)/16 + 1)
    w.tilemax = o; o = align256(o + 4LL * (px / 256 + (px + 1) / 16 + 4));
    w.total = o;
    return w;
}

void set_smem_attr(const void* kernel, size_t bytes) {
    // Not a stream operation; cheap after the first call.
    cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

template <int TABLE>
void fill_day_table(GvfTable<TABLE>& tab, const int32_t* dxdy, int second, int pitch) {
    for (int i = 0; i < SOLWEIG_GVF_DIRECTIONS * second; ++i) {
        tab.offs[i] = make_int2(dxdy[2 * i], dxdy[2 * i + 1]);
        tab.delta[i] = dxdy[2 * i] * pitch + dxdy[2 * i + 1];
    }
}

template <int TY, int FIRST, int SECOND, int TABLE>
void launch_day_gvf_ty(const SolweigScene& S, const SolweigHour* hours, int nhours, const DayGvfArgs& ga,
                       const GvfTable<TABLE>& tab, const float4* quads, const float* lup_first, float* gvf,
                       float* nosh, cudaStream_t st) {
    const size_t smem = sizeof(float4) * (size_t)(32 + 2 * ga.halo) * (TY + 2 * ga.halo);
    dim3 grid(blocks_for(S.cols, 32), blocks_for(S.rows, TY), nhours);
    if (S.has_water) {
        auto k = day_gvf_kernel<TY, FIRST, SECOND, TABLE, true>;
        set_smem_attr((const void*)k, smem);
        k<<<grid, dim3(32, TY), smem, st>>>(S, hours, ga, tab, quads, lup_first, gvf, nosh);
    } else {
        auto k = day_gvf_kernel<TY, FIRST, SECOND, TABLE, false>;
        set_smem_attr((const void*)k, smem);
        k<<<grid, dim3(32, TY), smem, st>>>(S, hours, ga, tab, quads, lup_first, gvf, nosh);
    }
}

template <int FIRST, int SECOND, int TABLE>
void launch_day_gvf(int ty, const SolweigScene& S, const SolweigHour* hours, int nhours, const DayGvfArgs& ga,
                    const GvfTable<TABLE>& tab, const float4* quads, const float* lup_first, float* gvf,
                    float* nosh, cudaStream_t st) {
    if (ty == 4) launch_day_gvf_ty<4, FIRST, SECOND, TABLE>(S, hours, nhours, ga, tab, quads, lup_first, gvf, nosh, st);
    else if (ty == 16) launch_day_gvf_ty<16, FIRST, SECOND, TABLE>(S, hours, nhours, ga, tab, quads, lup_first, gvf, nosh, st);
    else launch_day_gvf_ty<8, FIRST, SECOND, TABLE>(S, hours, nhours, ga, tab, quads, lup_first, gvf, nosh, st);
}

int launch_gemm(const uint32_t* masks, long long px, int patches, const __nv_bfloat16* b, int ncols, int nb,
                float* out, int* error, cudaStream_t st, int ctas_per_sm = 0, bool combined = false) {
    if (combined && gemm_pipe_smem_bytes(nb) <= 227 * 1024) {
        // the pipelined kernel: one CTA per SM (its shared memory)
        const size_t smem = gemm_pipe_smem_bytes(nb);
        set_smem_attr((const void*)patch_gemm_pipe_kernel, smem);
        int dev = 0, sms = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        const long long ntiles = (px + kARows - 1) / kARows;
        long long grid = sms > 0 ? sms : 1;
        if (grid > ntiles) grid = ntiles;
        GemmArgs g{masks, px, patches, b, ncols, nb, out, error, 1};
        patch_gemm_pipe_kernel<<<(unsigned)grid, kPipeThreads, smem, st>>>(g);
        SOLWEIG_CHECK_LAUNCH("patch_gemm_pipe_kernel");
        return SOLWEIG_OK;
    }
    const size_t smem = gemm_smem_bytes(nb, combined);
    SOLWEIG_CHECK_ARG(smem <= 227 * 1024, "patch contraction: %d weight columns need %zu bytes of shared memory",
                      ncols, smem);
    set_smem_attr((const void*)patch_gemm_kernel, smem);
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, patch_gemm_kernel, kARows, smem);
    if (per_sm < 1) per_sm = 1;
    if (ctas_per_sm > 0 && ctas_per_sm < per_sm) per_sm = ctas_per_sm;
    const long long ntiles = (px + kARows - 1) / kARows;
    long long grid = (long long)sms * per_sm;
    if (grid > ntiles) grid = ntiles;
    if (grid < 1) grid = 1;
    GemmArgs g{masks, px, patches, b, ncols, nb, out, error, combined ? 1 : 0};
    patch_gemm_kernel<<<(unsigned)grid, kARows, smem, st>>>(g);
    SOLWEIG_CHECK_LAUNCH("patch_gemm_kernel");
    return SOLWEIG_OK;
}

}  // namespace

}  // namespace solweig
