// Ground view factors (src/umep_solweig.py:583-663 gvf_2018a and :1400-1600
// sunonsurface_2018a).
//
// For every pixel, 18 search directions (azimuth 5, 25, ..., 345 degrees)
// walk `second` steps (22 for 1 m pixels) over four per-pixel fields: the
// shadow value, the emitted excess longwave Lup, the albedo and two bits
// (ground, sunlit wall).  The walk keeps f = running min of the ground bit, so
// f drops to 0 for good once the walk crosses a building; the reference also
// freezes a sample once it leaves the raster (its shifted copies are not
// cleared between steps).  After either event every further step adds the
// same increments, so the remaining steps are added in closed form.
//
// The fields are staged once per block in shared memory as one float4 per
// pixel (a (TX + 2H) x (TY + 2H) tile, H = second - 1) and every step of every
// direction is one 16-byte shared load; a warp's 32 lanes read 32 consecutive
// pixels of one tile row, which is conflict-free.
#pragma once
#include "common.cuh"

namespace solweig {

// Bits of the .w component of a GVF field quad.
constexpr int kQuadGround = 1;
constexpr int kQuadSunwall = 2;

struct GvfSums {
    float lup[5], alb[5], nosh[5];  // all, E, S, W, N  (sums over directions)
    float gvf_sum;
};

struct GvfScalars {
    float lwall;      // SBC*ewall*((Tgwall+Ta+273.15)^4 - (Ta+273.15)^4)
    float albedo_b;
    int first, second;
};

// Direction j (azimuth 5 + 20 j) belongs to E (0 <= az < 180), S (90..270),
// W (180..360) and N (>= 270 or < 90).
__device__ __forceinline__ unsigned gvf_direction_groups(int j) {
    const int az = 5 + 20 * j;
    unsigned g = 1u;  // all
    if (az < 180) g |= 2u;
    if (az >= 90 && az < 270) g |= 4u;
    if (az >= 180) g |= 8u;
    if (az >= 270 || az < 90) g |= 16u;
    return g;
}

// Walk all 18 directions for one pixel.  `sample(rr, cc)` returns the float4
// quad of an in-raster pixel; `lup_first(rr, cc)` returns the Lup used by
// direction 0 (differs from quad.y only for water pixels).
template <typename Sample, typename LupFirst>
__device__ __forceinline__ GvfSums gvf_walk(Sample sample, LupFirst lup_first, bool use_lup_first,
                                            int r, int c, int rows, int cols,
                                            const int2* __restrict__ offs, uint32_t face_mask,
                                            const float4 own, const GvfScalars g) {
    GvfSums out;
#pragma unroll
    for (int i = 0; i < 5; ++i) out.lup[i] = out.alb[i] = out.nosh[i] = 0.f;
    out.gvf_sum = 0.f;
    const float second = (float)g.second, first = (float)g.first;
    const bool own_ground = (__float_as_int(own.w) & kQuadGround) != 0;
    const float own_b = own_ground ? 1.f : 0.f;
    // Per-direction additive corrections of the reference (own pixel).
    const float corr_lup = own.y * (1.f - own_b);
    const float corr_alb = own.z * (1.f - own_b) * own.x;
    const float corr_nosh = own.z * (1.f - own_b);
    for (int j = 0; j < SOLWEIG_GVF_DIRECTIONS; ++j) {
        const int2* o = offs + j * g.second;
        float f = own_b;
        float t_sh = 0.f, t_lup = 0.f, t_alb = 0.f, t_albsh = 0.f;
        bool t_bu = false, t_sun = false;
        float s_sh = 0.f, s_lup = 0.f, s_albsh = 0.f, s_alb = 0.f;
        float s_wall = 0.f, s_lwall = 0.f, s_albwall = 0.f, s_albwall_nosh = 0.f;
        bool seen_sun = false, seen_wall = false;
        // snapshot after `first` steps
        float n_wall = 0.f, n_sh = 0.f, n_lwall = 0.f, n_lup = 0.f, n_albwall = 0.f, n_albsh = 0.f,
              n_albwall_nosh = 0.f, n_alb = 0.f;
        int n = 0;
        for (; n < g.second; ++n) {
            const int rr = r + o[n].x, cc = c + o[n].y;
            const bool inside = in_raster(rr, cc, rows, cols);
            if (inside) {
                const float4 q = sample(rr, cc);
                t_sh = q.x;
                t_lup = (use_lup_first && j == 0) ? lup_first(rr, cc) : q.y;
                t_alb = q.z;
                t_albsh = q.z * q.x;
                const int bits = __float_as_int(q.w);
                t_bu = (bits & kQuadGround) != 0;
                t_sun = (bits & kQuadSunwall) != 0;
            }
            if (!t_bu) f = 0.f;
            // f is 0 or 1, so t * f is either t or 0.
            if (f != 0.f) {
                s_sh += t_sh;
                s_lup += t_lup;
                s_albsh += t_albsh;
                s_alb += t_alb;
                seen_sun = seen_sun || t_sun;
            } else {
                seen_wall = true;
            }
            if (seen_sun) {
                s_lwall += g.lwall;
                s_albwall += g.albedo_b;
                s_wall += 1.f;
            }
            if (seen_wall) s_albwall_nosh += g.albedo_b;
            if (n + 1 <= g.first) {
                n_wall = s_wall; n_sh = s_sh; n_lwall = s_lwall; n_lup = s_lup;
                n_albwall = s_albwall; n_albsh = s_albsh; n_albwall_nosh = s_albwall_nosh;
                n_alb = s_alb;
            }
            // From here on every step adds the same increments: f stayed 0, or
            // the sample left the raster (values frozen).  Finish in closed form
            // once the `first` snapshot is taken.
            if ((f == 0.f || !inside) && n + 1 >= g.first) {
                const float rest = (float)(g.second - 1 - n);
                if (f != 0.f) {
                    s_sh += rest * t_sh;
                    s_lup += rest * t_lup;
                    s_albsh += rest * t_albsh;
                    s_alb += rest * t_alb;
                }
                if (seen_sun) {
                    s_lwall += rest * g.lwall;
                    s_albwall += rest * g.albedo_b;
                    s_wall += rest;
                }
                if (seen_wall) s_albwall_nosh += rest * g.albedo_b;
                break;
            }
        }
        const bool sun_near = n_wall > 0.f, wall_near = n_albwall_nosh > 0.f;
        const bool sun_far = s_wall > 0.f, wall_far = s_albwall_nosh > 0.f;
        // Wall faces turned away from this direction drop their wall terms when
        // every step saw a sunlit wall (keep == 1 in the reference).
        if (s_wall == second && ((face_mask >> j) & 1u)) {
            s_wall = 0.f;
            s_lwall = 0.f;
            s_albwall = 0.f;
        }
        float gvf2 = sun_far ? (s_wall + s_sh) / (second + 1.f) : s_sh / second;
        if (gvf2 > 1.f) gvf2 = 1.f;
        const float lup1 = sun_near ? (n_lwall + n_lup) / (first + 1.f) : n_lup / first;
        const float lup2 = sun_far ? (s_lwall + s_lup) / (second + 1.f) : s_lup / second;
        const float alb1 = sun_near ? (n_albwall + n_albsh) / (first + 1.f) : n_albsh / first;
        const float alb2 = sun_far ? (s_albwall + s_albsh) / (second + 1.f) : s_albsh / second;
        const float nosh1 = wall_near ? (n_albwall_nosh + n_alb) / (first + 1.f) : n_alb / first;
        const float nosh2 = wall_far ? (s_albwall_nosh + s_alb) / second : s_alb / second;
        const float d_lup = (lup1 * 0.5f + lup2 * 0.4f) / 0.9f + corr_lup;
        const float d_alb = (alb1 * 0.5f + alb2 * 0.4f) / 0.9f + corr_alb;
        const float d_nosh = ((nosh1 * 0.5f + nosh2 * 0.4f) / 0.9f) * own_b + corr_nosh;
        const unsigned groups = gvf_direction_groups(j);
#pragma unroll
        for (int k = 0; k < 5; ++k)
            if (groups & (1u << k)) {
                out.lup[k] += d_lup;
                out.alb[k] += d_alb;
                out.nosh[k] += d_nosh;
            }
        out.gvf_sum += gvf2;
    }
    return out;
}

// Cooperative load of the block's quad tile (with halo) into shared memory.
__device__ __forceinline__ void load_quad_tile(float4* tile, int pitch, int tile_rows,
                                               const float4* __restrict__ quad, int rows, int cols,
                                               int row0, int col0) {
    const int n = pitch * tile_rows;
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    const int nthreads = blockDim.x * blockDim.y;
    for (int i = tid; i < n; i += nthreads) {
        const int tr = i / pitch, tc = i - tr * pitch;
        const int rr = row0 + tr, cc = col0 + tc;
        tile[i] = in_raster(rr, cc, rows, cols) ? __ldg(&quad[(long long)rr * cols + cc])
                                                : make_float4(0.f, 0.f, 0.f, 0.f);
    }
}

}  // namespace solweig
