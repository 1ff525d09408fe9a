// The shadow sweep: building and vegetation shadows along one sun ray.
//
// For every pixel p and ray step k the reference (src/umep_solweig.py:2201-2406)
// shifts the DSM / canopy / trunk rasters by the step offset, subtracts the
// step height dz_k (all float64) and accumulates:
//   f      = max(dsm_p, max_k(dsm[p+off_k] - dz_k))          building top seen
//   topmax = max(vegdem_p, max_k(vegdem[p+off_k] - dz_k))    canopy top seen
//   shadowed_k = f > dsm_p
//   veg    |= 1 <= #{top-dz_k, bot-dz_k, top-dz_{k-1}, bot-dz_{k-1} > dsm_p} <= 3,
//             cleared whenever shadowed_k
//   ever   |= veg
// Samples outside the raster read as exactly 0 (no dz subtracted).
//
// The per-pixel loop below evaluates these recurrences in the same float64
// operations, so every mask is bit-identical to the reference, and stops early
// when the remaining steps provably change nothing:
//   * hmax - dz_{k-1} < dsm_p (exactly) -> no later sample can rise above the
//     pixel (and, for wall pixels, hmax - dz_k <= topmax so the canopy top is
//     final); only taken when dsm_p >= 0 (and topmax >= 0), so the zero-valued
//     samples beyond the raster edge could not change anything either;
//   * a sample without canopy (top, trunk <= 0) skips the canopy compares
//     (with dsm_p >= 0 and topmax >= 0 they cannot change anything);
//   * shadowed and not a wall pixel -> every output is final;
//   * shadowed wall pixel with f - dsm_p >= wall -> wallsun is already 0;
//   * with a ray-ceiling plane (ceiling.cuh), every 4th step from step 4 on:
//     ceiling(q_k) - dz_{k-1} (rounded up) < dsm_p bounds every later
//     sample's h - dz_{j-1} below the pixel (dsm_p >= 0; for wall pixels
//     also <= topmax >= 0), so nothing further can change;
//   * (packed walk) at the same steps, window maximum(q_k) - dz_{k-1}
//     (rounded up) <= dsm_p bounds the next kCeilSkip samples' h - dz_{j-1}
//     by the pixel: none of their compares is above it and f cannot grow, so
//     the walk skips them when, for a wall pixel, the bound is also <= topmax
//     (the canopy top seen stays final); only the carried flags move: ever
//     picks up veg when unshadowed, as each step would.
// Once a sample leaves the raster it never re-enters (the offsets grow
// monotonically), so the first outside step is applied and the loop ends.
#pragma once
#include "common.cuh"

namespace solweig {

struct ShadowResult {
    double f, topmax;
    bool shadowed, veg, ever;
};

// Height samples of the sweep: the three float64 rasters ...
struct GeoF64 {
    const double* __restrict__ dsm;
    const double* __restrict__ top;
    const double* __restrict__ bot;
    __device__ __forceinline__ void load(long long q, bool vegetation, double& a, double& t, double& b) const {
        a = __ldg(&dsm[q]);
        if (vegetation) {
            t = __ldg(&top[q]);
            b = __ldg(&bot[q]);
        }
    }
};

// ... or, when every value of all three is exactly representable in float32,
// one interleaved (dsm, canopy, trunk, 0) float4 per pixel: a single 16-byte
// load per step, widened to float64 exactly, so every compare is unchanged.
struct GeoF32x4 {
    const float4* __restrict__ geo;
    __device__ __forceinline__ void load(long long q, bool, double& a, double& t, double& b) const {
        const float4 v = __ldg(&geo[q]);
        a = v.x;
        t = v.y;
        b = v.z;
    }
};

// Walk the ray for pixel (r, c).  `is_wall` enables the wall-specific
// continuation rules; `hmax` = max over the raster of dsm, vegdem and vegdem2.
template <typename Geo>
__device__ __forceinline__ ShadowResult shadow_walk_geo(
    const Geo& geo, int rows, int cols, int r, int c, double a, double top_p, bool bush, double wall,
    const int2* __restrict__ ray, const double* __restrict__ dz, int steps, double hmax,
    bool vegetation, const float2* __restrict__ ceiling = nullptr) {
    ShadowResult s;
    s.f = a;
    s.topmax = top_p;
    s.shadowed = false;
    s.veg = bush;
    s.ever = false;
    const bool is_wall = wall > 0.0;
    // dz_prev >= clear  =>  hmax - dz_prev < a in exact arithmetic (the
    // threshold is one ulp above the rounded difference), so no later sample
    // of any of the three rasters can rise above the pixel.
    const double clear = a >= 0.0 ? nextafter(hmax - a, __longlong_as_double(0x7ff0000000000000ll))
                                  : __longlong_as_double(0x7ff0000000000000ll);
    double dz_prev = 0.0;
    int k = 0;
    for (; k < steps; ++k) {
        const int2 o = __ldg(&ray[k]);
        const double dzk = __ldg(&dz[k]);
        const int rr = r + o.x, cc = c + o.y;
        if (!in_raster(rr, cc, rows, cols)) break;
        const long long q = (long long)rr * cols + cc;
        // Early exits that cannot change any output.
        if (dz_prev >= clear && (!is_wall || (s.topmax >= 0.0 && hmax - dzk <= s.topmax))) {
            k = steps;  // nothing further can change; no outside fix-up needed
            break;
        }
        if (ceiling != nullptr && k >= 4 && (k & 3) == 0) {
            const double e = __dsub_ru((double)__ldg(&ceiling[q]).x, dz_prev);
            if (a >= 0.0 && e < a && (!is_wall || (s.topmax >= 0.0 && e <= s.topmax))) {
                k = steps;
                break;
            }
        }
        double hq, tq = 0.0, bq = 0.0;
        geo.load(q, vegetation, hq, tq, bq);
        const double aq = hq - dzk;
        s.f = fmax(s.f, aq);
        s.shadowed = s.f > a;
        if (vegetation) {
            if (tq <= 0.0 && bq <= 0.0 && a >= 0.0 && s.topmax >= 0.0) {
                // No canopy at this sample: its shifted tops are <= 0 <= a and
                // cannot raise topmax, so only the carried flags move.
                if (s.shadowed) s.veg = false;
                else s.ever = s.ever || s.veg;
            } else {
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
        }
        if (s.shadowed && (!is_wall || s.f - a >= wall)) {
            k = steps;
            break;
        }
        dz_prev = dzk;
    }
    if (k < steps) {
        // First step whose sample is outside the raster: all shifted values are 0.
        s.f = fmax(s.f, 0.0);
        s.shadowed = s.f > a;
        if (vegetation) {
            s.topmax = fmax(s.topmax, 0.0);
            if (s.shadowed) s.veg = false;
            s.ever = s.ever || s.veg;
        }
    }
    return s;
}

// The same walk over the packed float4 geometry, for a ray known to stay in
// the raster for `kend` steps (the first step outside, or `steps`): no
// per-step bounds checks, linear sample offsets, and only the DSM height is
// widened to float64 at a sample without canopy (tq, bq <= 0 compare the
// same in float32).  Results are identical to shadow_walk_geo.
//
// The steps run in unrolled groups of four aligned at step 0, so the
// ray-ceiling test (steps 4, 8, ...) is the first step of a group and costs
// no per-step test.  With REC the hour's steps come as 16-byte records
// {linear offset o.x * cols + o.y, dz bit pattern} (one uniform load per
// step, ray_records_block); otherwise from the (dx, dy) and dz tables.
template <bool REC, bool SKIP = true>
__device__ __forceinline__ ShadowResult shadow_walk_packed(
    const float4* __restrict__ geo, int cols, long long p, double a, double top_p, bool bush, double wall,
    const int2* __restrict__ ray, const double* __restrict__ dz, const longlong2* __restrict__ rec, int steps,
    int kend, double hmax, const float2* __restrict__ ceiling) {
    ShadowResult s;
    s.f = a;
    s.topmax = top_p;
    s.shadowed = false;
    s.veg = bush;
    s.ever = false;
    const bool is_wall = wall > 0.0;
    const bool nonneg = a >= 0.0;
    const double clear = nonneg ? nextafter(hmax - a, __longlong_as_double(0x7ff0000000000000ll))
                                : __longlong_as_double(0x7ff0000000000000ll);
    const float4* __restrict__ gp = geo + p;
    const float2* __restrict__ cp = ceiling != nullptr ? ceiling + p : nullptr;
    double dz_prev = 0.0;
    bool final = false;
    int k = 0;
    while (k < kend) {
#pragma unroll
        for (int u = 0; u < 4; ++u) {  // u == k % 4
            if (k >= kend) break;
            long long off;
            double dzk;
            if (REC) {
                const longlong2 r = __ldg(rec + k);
                off = r.x;
                dzk = __longlong_as_double(r.y);
            } else {
                const int2 o = __ldg(&ray[k]);
                dzk = __ldg(&dz[k]);
                off = (long long)o.x * cols + o.y;
            }
            if (dz_prev >= clear && (!is_wall || (s.topmax >= 0.0 && hmax - dzk <= s.topmax))) {
                final = true;
                break;
            }
            if (u == 0 && cp != nullptr && k >= 4) {
                const float2 cm = __ldg(cp + off);
                const double e = __dsub_ru((double)cm.x, dz_prev);
                if (nonneg && e < a && (!is_wall || (s.topmax >= 0.0 && e <= s.topmax))) {
                    final = true;
                    break;
                }
                const double em = __dsub_ru((double)cm.y, dz_prev);
                if (SKIP && nonneg && k + kCeilSkip <= kend && em <= a && (!is_wall || em <= s.topmax)) {
                    // steps k .. k + kCeilSkip - 1 change nothing but the carried flags
                    s.ever = s.ever || s.veg;
                    k += kCeilSkip;
                    dz_prev = REC ? __longlong_as_double(__ldg(rec + k - 1).y) : __ldg(&dz[k - 1]);
                    break;  // the next group starts at k (still a multiple of 4)
                }
            }
            const float4 v = __ldg(gp + off);
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
            if (s.shadowed && (!is_wall || s.f - a >= wall)) {
                final = true;
                break;
            }
            dz_prev = dzk;
            ++k;
        }
        if (final) break;
    }
    if (!final && k < steps) {
        // First step whose sample is outside the raster: all shifted values are 0.
        s.f = fmax(s.f, 0.0);
        s.shadowed = s.f > a;
        s.topmax = fmax(s.topmax, 0.0);
        if (s.shadowed) s.veg = false;
        s.ever = s.ever || s.veg;
    }
    return s;
}

// Step records of one hour's ray for shadow_walk_packed<true>: rec[k] =
// {o_k.x * cols + o_k.y, dz_k as a 64-bit pattern} for k < K, by one block.
__device__ __forceinline__ void ray_records_block(const int2* __restrict__ ray, const double* __restrict__ dz,
                                                  int K, int cols, longlong2* __restrict__ rec) {
    for (int k = threadIdx.x; k < K; k += blockDim.x) {
        const int2 o = __ldg(&ray[k]);
        rec[k] = make_longlong2((long long)o.x * cols + o.y, __double_as_longlong(__ldg(&dz[k])));
    }
}

// Per hour, the first step at which the ray from row r (column c) leaves the
// raster: exits[r] for the rows, exits[rows + c] for the columns (`steps`
// when it never does).  The offsets of a sun ray are monotone along both
// axes, so the steps inside form a prefix found by bisection; a table whose
// offsets are not monotone is scanned linearly.
__device__ __forceinline__ int first_outside(const int2* __restrict__ ray, int steps, bool row_axis, int pos,
                                             int extent, bool monotone) {
    auto inside = [&](int k) {
        const int2 o = __ldg(&ray[k]);
        const int v = pos + (row_axis ? o.x : o.y);
        return v >= 0 && v < extent;
    };
    if (!monotone) {
        for (int k = 0; k < steps; ++k)
            if (!inside(k)) return k;
        return steps;
    }
    int lo = 0, hi = steps;  // inside on [0, lo), answer in [lo, hi]
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (inside(mid)) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// first_outside of every row (exits[r]) and column (exits[rows + c]) of a
// rows x cols raster for one ray table, by one block: the offsets are checked
// for monotony along each axis first (bisection needs it).
__device__ __forceinline__ void ray_exits_block(const int2* __restrict__ ray, int K, int rows, int cols,
                                                int* __restrict__ exits) {
    int xi = 1, xd = 1, yi = 1, yd = 1;
    for (int k = 1 + threadIdx.x; k < K; k += blockDim.x) {
        const int2 o = __ldg(&ray[k]), q = __ldg(&ray[k - 1]);
        xi &= o.x >= q.x;
        xd &= o.x <= q.x;
        yi &= o.y >= q.y;
        yd &= o.y <= q.y;
    }
    const int axi = __syncthreads_and(xi), axd = __syncthreads_and(xd);
    const int ayi = __syncthreads_and(yi), ayd = __syncthreads_and(yd);
    const bool mx = axi || axd, my = ayi || ayd;
    for (int i = threadIdx.x; i < rows + cols; i += blockDim.x)
        exits[i] = i < rows ? first_outside(ray, K, true, i, rows, mx)
                            : first_outside(ray, K, false, i - rows, cols, my);
}

__device__ __forceinline__ ShadowResult shadow_walk(
    const double* __restrict__ dsm, const double* __restrict__ top, const double* __restrict__ bot,
    int rows, int cols, int r, int c, double a, double top_p, bool bush, double wall,
    const int2* __restrict__ ray, const double* __restrict__ dz, int steps, double hmax,
    bool vegetation) {
    return shadow_walk_geo(GeoF64{dsm, top, bot}, rows, cols, r, c, a, top_p, bush, wall, ray, dz, steps, hmax,
                           vegetation);
}

// Self-shadowed wall faces (facesh) for the sun window (low, high, middle).
__device__ __forceinline__ double self_shadow_face(double aspect, double wallbol, double low,
                                                   double high, int middle) {
    return middle ? (double)(aspect < low || aspect >= high) - wallbol + 1.0
                  : 1.0 - (double)(aspect > low || aspect <= high);
}

}  // namespace solweig
