// Lean ground-view-factor walk for the hourly step (the 15 planes the step
// needs: Lup, albedo, albedo-without-shadow for all / E / S / W / N).
//
// Same recurrences as gvf_walk (gvf.cuh, which also produces gvfSum and
// gvfNorm for the standalone entry point), restructured for throughput:
//   * the shared-memory tile address of every (direction, step) offset is
//     precomputed once per block, so a step is one 16-byte shared load;
//   * blocks whose halo tile lies inside the raster (all but a border band of
//     `second` pixels) take a path without per-step bounds checks;
//   * the wall terms of a step only depend on whether a sunlit wall / any
//     wall has been seen, so they are kept as integer step counts and scaled
//     once per direction;
//   * a walk stops at the first building (f = 0) or raster exit and adds the
//     remaining, identical steps in closed form.
#pragma once
#include "gvf.cuh"

namespace solweig {

struct GvfDir {
    float lup, alb, nosh;
};

// One direction for one pixel.  `tile` points at the pixel's own cell;
// `delta[n]` is the tile-address offset of step n.  Interior: no bounds checks.
template <bool Interior>
__device__ __forceinline__ GvfDir gvf_direction(const float4* __restrict__ tile,
                                                const int* __restrict__ delta,
                                                const int2* __restrict__ offs, int r, int c,
                                                int rows, int cols, bool own_ground, int first,
                                                int second, float inv_first, float inv_first1,
                                                float inv_second, float inv_second1, float lwall,
                                                float albedo_b, bool face) {
    float s_lup = 0.f, s_albsh = 0.f, s_alb = 0.f;
    float n_lup = 0.f, n_albsh = 0.f, n_alb = 0.f;  // sums after step first-1
    int n_sun = 0, n_sun_first = 0;                 // steps with a sunlit wall seen
    bool seen_sun = false;
    int hit = second;  // first step with f = 0 (second = never)
    bool f = own_ground;
    float4 q = make_float4(0.f, 0.f, 0.f, 0.f);
    for (int n = 0; n < second; ++n) {
        bool inside = true;
        if (!Interior) {
            const int2 o = offs[n];
            inside = in_raster(r + o.x, c + o.y, rows, cols);
        }
        if (inside) q = tile[delta[n]];
        const int bits = __float_as_int(q.w);
        if (!(bits & kQuadGround)) f = false;
        if (!f) {
            hit = n;
            break;
        }
        s_lup += q.y;
        s_albsh = fmaf(q.z, q.x, s_albsh);
        s_alb += q.z;
        seen_sun = seen_sun || (bits & kQuadSunwall);
        n_sun += seen_sun ? 1 : 0;
        if (n + 1 == first) {
            n_lup = s_lup; n_albsh = s_albsh; n_alb = s_alb; n_sun_first = n_sun;
        }
        if (!Interior && !inside) {
            // The sample left the raster: it stays frozen, so the remaining
            // steps repeat this one exactly.
            if (n + 1 < first) {
                const int k = first - 1 - n;
                n_lup = s_lup + k * q.y;
                n_albsh = s_albsh + k * (q.z * q.x);
                n_alb = s_alb + k * q.z;
                n_sun_first = n_sun + (seen_sun ? k : 0);
            }
            const int rest = second - 1 - n;
            s_lup += rest * q.y;
            s_albsh += rest * (q.z * q.x);
            s_alb += rest * q.z;
            n_sun += seen_sun ? rest : 0;
            break;
        }
    }
    if (hit < second) {
        // f = 0 from step `hit` on: the sunlit-wall flag is frozen and every
        // remaining step sees a wall.
        if (hit < first) {
            n_lup = s_lup; n_albsh = s_albsh; n_alb = s_alb;
            n_sun_first = n_sun + (seen_sun ? first - hit : 0);
        }
        n_sun += seen_sun ? second - hit : 0;
    }
    const int n_wall = second - hit;                       // steps with a wall seen
    const int n_wall_first = first > hit ? first - hit : 0;
    float s_wall = (float)n_sun;
    const bool sun_far = n_sun > 0, wall_far = n_wall > 0;
    const bool sun_near = n_sun_first > 0, wall_near = n_wall_first > 0;
    float s_lwall = s_wall * lwall, s_albwall = s_wall * albedo_b;
    if (s_wall == (float)second && face) {
        s_lwall = 0.f;
        s_albwall = 0.f;
    }
    const float nn_sun = (float)n_sun_first;
    const float lup1 = sun_near ? (nn_sun * lwall + n_lup) * inv_first1 : n_lup * inv_first;
    const float lup2 = sun_far ? (s_lwall + s_lup) * inv_second1 : s_lup * inv_second;
    const float alb1 = sun_near ? (nn_sun * albedo_b + n_albsh) * inv_first1 : n_albsh * inv_first;
    const float alb2 = sun_far ? (s_albwall + s_albsh) * inv_second1 : s_albsh * inv_second;
    const float nosh1 = wall_near ? ((float)n_wall_first * albedo_b + n_alb) * inv_first1 : n_alb * inv_first;
    const float nosh2 = wall_far ? ((float)n_wall * albedo_b + s_alb) * inv_second : s_alb * inv_second;
    GvfDir d;
    d.lup = (lup1 * 0.5f + lup2 * 0.4f) * (1.f / 0.9f);
    d.alb = (alb1 * 0.5f + alb2 * 0.4f) * (1.f / 0.9f);
    d.nosh = (nosh1 * 0.5f + nosh2 * 0.4f) * (1.f / 0.9f);
    return d;
}

}  // namespace solweig

namespace solweig {

// Step offsets of the 18 directions for a compile-time walk length: tile
// address deltas (for the block's tile pitch) and raster offsets, passed as a
// kernel parameter so every (direction, step) lookup is a uniform constant-bank
// read instead of a shared-memory load.
template <int SECOND>
struct GvfTable {
    int delta[SOLWEIG_GVF_DIRECTIONS * SECOND];
    int2 offs[SOLWEIG_GVF_DIRECTIONS * SECOND];
};

// gvf_direction with the walk length and the `first` snapshot fixed at
// compile time (the 1 m default: first = 1, second = 22), fully unrolled.
template <bool Interior, int FIRST, int SECOND>
__device__ __forceinline__ GvfDir gvf_direction_fixed(const float4* __restrict__ tile,
                                                      const int* delta, const int2* offs, int r,
                                                      int c, int rows, int cols, bool own_ground,
                                                      float lwall, float albedo_b, bool face) {
    float s_lup = 0.f, s_albsh = 0.f, s_alb = 0.f;
    float n_lup = 0.f, n_albsh = 0.f, n_alb = 0.f;
    int n_sun = 0, n_sun_first = 0;
    bool seen_sun = false;
    int hit = SECOND;
    float4 q = make_float4(0.f, 0.f, 0.f, 0.f);
    bool frozen = false;
    if (own_ground) {
#pragma unroll
        for (int n = 0; n < SECOND; ++n) {
            bool inside = true;
            if (!Interior) {
                const int2 o = offs[n];
                inside = in_raster(r + o.x, c + o.y, rows, cols);
            }
            if (inside) q = tile[delta[n]];
            const int bits = __float_as_int(q.w);
            if (!(bits & kQuadGround)) {
                hit = n;
                break;
            }
            s_lup += q.y;
            s_albsh = fmaf(q.z, q.x, s_albsh);
            s_alb += q.z;
            seen_sun = seen_sun || (bits & kQuadSunwall);
            n_sun += seen_sun ? 1 : 0;
            if (n + 1 == FIRST) {
                n_lup = s_lup; n_albsh = s_albsh; n_alb = s_alb; n_sun_first = n_sun;
            }
            if (!Interior && !inside) {
                if (n + 1 < FIRST) {
                    const int k = FIRST - 1 - n;
                    n_lup = s_lup + k * q.y;
                    n_albsh = s_albsh + k * (q.z * q.x);
                    n_alb = s_alb + k * q.z;
                    n_sun_first = n_sun + (seen_sun ? k : 0);
                }
                const int rest = SECOND - 1 - n;
                s_lup += rest * q.y;
                s_albsh += rest * (q.z * q.x);
                s_alb += rest * q.z;
                n_sun += seen_sun ? rest : 0;
                frozen = true;
                break;
            }
        }
    } else {
        hit = 0;
    }
    (void)frozen;
    if (hit < SECOND) {
        if (hit < FIRST) {
            n_lup = s_lup; n_albsh = s_albsh; n_alb = s_alb;
            n_sun_first = n_sun + (seen_sun ? FIRST - hit : 0);
        }
        n_sun += seen_sun ? SECOND - hit : 0;
    }
    const int n_wall = SECOND - hit;
    const int n_wall_first = FIRST > hit ? FIRST - hit : 0;
    const float s_wall = (float)n_sun;
    const bool sun_far = n_sun > 0, wall_far = n_wall > 0;
    const bool sun_near = n_sun_first > 0, wall_near = n_wall_first > 0;
    float s_lwall = s_wall * lwall, s_albwall = s_wall * albedo_b;
    if (n_sun == SECOND && face) {
        s_lwall = 0.f;
        s_albwall = 0.f;
    }
    constexpr float inv_first = 1.f / FIRST, inv_first1 = 1.f / (FIRST + 1);
    constexpr float inv_second = 1.f / SECOND, inv_second1 = 1.f / (SECOND + 1);
    const float nn_sun = (float)n_sun_first;
    const float lup1 = sun_near ? (nn_sun * lwall + n_lup) * inv_first1 : n_lup * inv_first;
    const float lup2 = sun_far ? (s_lwall + s_lup) * inv_second1 : s_lup * inv_second;
    const float alb1 = sun_near ? (nn_sun * albedo_b + n_albsh) * inv_first1 : n_albsh * inv_first;
    const float alb2 = sun_far ? (s_albwall + s_albsh) * inv_second1 : s_albsh * inv_second;
    const float nosh1 = wall_near ? ((float)n_wall_first * albedo_b + n_alb) * inv_first1 : n_alb * inv_first;
    const float nosh2 = wall_far ? ((float)n_wall * albedo_b + s_alb) * inv_second : s_alb * inv_second;
    GvfDir d;
    d.lup = (lup1 * 0.5f + lup2 * 0.4f) * (1.f / 0.9f);
    d.alb = (alb1 * 0.5f + alb2 * 0.4f) * (1.f / 0.9f);
    d.nosh = (nosh1 * 0.5f + nosh2 * 0.4f) * (1.f / 0.9f);
    return d;
}

}  // namespace solweig
