// Per-pixel pieces of one SOLWEIG hour shared by the per-hour step
// (step.cu) and the batched day (day.cu).
#pragma once
#include "gvf.cuh"
#include "shadow.cuh"

namespace solweig {

// Ground temperature amplitude wave of the hour (before the water override).
__device__ __forceinline__ double ground_tg(const SolweigScene& S, const SolweigHour& h,
                                            long long p) {
    const double amp = (double)S.tgk[p] * h.altmax + (double)S.tstart[p];
    const double phase =
        ((h.dectime_frac - h.snup / 24.0) / ((double)S.tmaxlst[p] / 24.0 - h.snup / 24.0)) * kPi / 2.0;
    double tg = amp * sin(phase) * h.ci_tgg;
    if (S.landcover == 1 && tg < 0.0) tg = 0.0;
    return tg;
}

__device__ __forceinline__ double lup_excess(double emis, double tg, double shadow, double ta) {
    return kSBC * emis * pow4(tg * shadow + ta + 273.15) - kSBC * emis * pow4(ta + 273.15);
}

// The quad of one pixel-hour from its walk result: the wall's sunlit height
// (only for the sunlit-wall bit of the GVF), the shadow and the Lup excess
// (also written to lup_first, when given, before the water override).
// Shared by the raster and the window sweeps.
__device__ __forceinline__ float4 quad_from_walk(const SolweigScene& S, const SolweigHour& h, long long p,
                                                 double a, double wall, uint8_t fl, const ShadowResult& s,
                                                 float* __restrict__ lup_first) {
    const double wallbol = wall > 0.0 ? 1.0 : 0.0;
    const double facesh = self_shadow_face(S.aspect[p], wallbol, h.ray_low, h.ray_high, h.ray_middle);
    double wallsun = wall - (s.f - a);
    if (wallsun < 0.0) wallsun = 0.0;
    if (facesh == 1.0) wallsun = 0.0;
    const double wallsh = wall - wallsun;
    double wallshve = (s.topmax - a) * (s.veg ? 1.0 : 0.0) * wallbol - wallsh;
    if (wallshve < 0.0) wallshve = 0.0;
    if (wallshve > wall) wallshve = wall;
    wallsun = wallsun - wallshve;
    if (wallsun < 0.0) wallsun = 0.0;
    // (wallsun / wall * ground) == 1 of the reference: a correctly rounded
    // quotient of two finite doubles is exactly 1 only when they are equal,
    // and 0 / 0 (no wall) is NaN, so no division is needed.
    const bool sunwall = (fl & 1) && wall > 0.0 && wallsun == wall;
    const double sh = s.shadowed ? 0.0 : 1.0;
    const double vegsh = s.veg ? 0.0 : 1.0;
    const double shadow = (double)(float)(sh - (1.0 - vegsh) * (1.0 - h.psi));
    double tg = ground_tg(S, h, p);
    const double emis = S.emis[p];
    if (lup_first) lup_first[p] = (float)lup_excess(emis, tg, shadow, h.ta);
    if (S.has_water && (fl & 4)) tg = h.twater - h.ta;
    const float lup = (float)lup_excess(emis, tg, shadow, h.ta);
    return make_float4((float)shadow, lup, S.alb[p],
                       __int_as_float((fl & 1 ? kQuadGround : 0) | (sunwall ? kQuadSunwall : 0)));
}

// Shadow sweep of pixel (r, c) for hour h and the per-pixel GVF inputs: the
// float4 quad (shadow, Lup, albedo, ground|sunwall bits; also returned) and,
// for scenes with water, the Lup of the first GVF search direction.
// `exits` (optional): the hour's first-outside step of every row and column
// (first_outside); with the packed geometry the walk then needs no bounds checks.
// REC (with exits and the packed geometry): the walk reads the hour's step
// records `rec` (ray_records_block) instead of the (dx, dy) and dz tables.
template <bool REC = false>
__device__ __forceinline__ float4 shadow_quad_pixel(const SolweigScene& S, const SolweigHour& h, int r, int c,
                                                  float4* __restrict__ quad, float* __restrict__ lup_first,
                                                  const float2* __restrict__ ceiling = nullptr,
                                                  const int* __restrict__ exits = nullptr,
                                                  const longlong2* __restrict__ rec = nullptr) {
    const long long p = (long long)r * S.cols + c;
    const double a = S.dsm[p];
    const double wall = S.walls[p];
    const uint8_t fl = S.flags[p];
    const int2* ray = reinterpret_cast<const int2*>(h.ray_dxdy);
    ShadowResult s;
    if (S.geo32 && exits) {
        const int kend = min(h.steps, min(__ldg(&exits[r]), __ldg(&exits[S.rows + c])));
        const float4* geo = reinterpret_cast<const float4*>(S.geo32);
        s = shadow_walk_packed<REC>(geo, S.cols, p, a, S.vegdem[p], (fl & 2) != 0, wall, ray, h.ray_dz, rec,
                                    h.steps, kend, S.hmax, ceiling);
    } else if (S.geo32) {
        s = shadow_walk_geo(GeoF32x4{reinterpret_cast<const float4*>(S.geo32)}, S.rows, S.cols, r, c, a,
                            S.vegdem[p], (fl & 2) != 0, wall, ray, h.ray_dz, h.steps, S.hmax, true, ceiling);
    } else {
        s = shadow_walk_geo(GeoF64{S.dsm, S.vegdem, S.vegdem2}, S.rows, S.cols, r, c, a, S.vegdem[p],
                            (fl & 2) != 0, wall, ray, h.ray_dz, h.steps, S.hmax, true, ceiling);
    }
    const float4 q = quad_from_walk(S, h, p, a, wall, fl, s, lup_first);
    quad[p] = q;
    return q;
}

}  // namespace solweig
