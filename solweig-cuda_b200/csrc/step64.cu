// The hourly SOLWEIG step with float64 radiation: the reference's
// `--dtype float64` switch (run.py:27), which recompiles its gvf.cu,
// shortwave.cu, longwave.cu and flux.cu kernels with Real = double
// (src/runtime.py:43-49, src/model.py:382-620, :731).
//
//  K1 step64_fields_kernel     shadow sweep (the float32 step's walk over the
//                              float64 rasters: the same masks) and the
//                              per-pixel GVF inputs in float64: shadow, Lup
//                              excess (before and after the water override),
//                              albedo * shadow and the ground / sunlit-wall bits
//  K2 step64_gvf_kernel        the 18 search directions of gvf_2018a /
//                              sunonsurface_2018a (src/umep_solweig.py:583-663,
//                              :1400-1600), every step added in order
//  K3 step64_radiation_kernel  wave delay, F_sh, Kup, Kdown, Kside and the
//                              anisotropic longwave (Kside_veg_v2022a :666-911,
//                              Lcyl_v2022a :946-1028), Tmrt (:345-360) and UTCI
//
// Everything per pixel is float64 and the patch sums run over every patch in
// patch order, with products grouped as the reference's expressions group
// them.  This file is compiled with --fmad=false (as the reference compiles
// its kernels, src/runtime.py:11), so no multiply-add is contracted.  UTCI is
// evaluated from the float32-rounded Tmrt and air temperature, as
// utci_calculator casts its inputs (src/utci.py:8-12).
#include "hour.cuh"
#include "radiation.cuh"

namespace solweig {

constexpr int kStep64BX = 32, kStep64BY = 4;

// Scratch planes [SOLWEIG_SCRATCH64_PLANES][pixels] float64.
enum Scratch64 : int {
    kS64Shadow = 0,    // sh - (1 - vegsh)(1 - psi)
    kS64Lup = 1,       // Lup excess after the water override
    kS64LupFirst = 2,  // Lup excess before it (first search direction)
    kS64AlbSh = 3,     // albedo * shadow
    kS64Bits = 4,      // 1 = ground, 2 = sunlit wall (small integers)
    kS64Gvf = 5,       // 15 planes: Lup, albedo, albedo without shadow x (all, E, S, W, N)
};

struct GvfOffsets64 {
    int2 offs[SOLWEIG_GVF_DIRECTIONS * SOLWEIG_GVF_MAX_STEPS];
};

__global__ void __launch_bounds__(kStep64BX* kStep64BY) step64_fields_kernel(
    SolweigScene S, const SolweigHour* __restrict__ hours, int hour, double* __restrict__ sc) {
    const SolweigHour& h = hours[hour];
    if (!h.daytime) return;
    const int c = blockIdx.x * kStep64BX + threadIdx.x;
    const int r = blockIdx.y * kStep64BY + threadIdx.y;
    if (r >= S.rows || c >= S.cols) return;
    const long long n = (long long)S.rows * S.cols;
    const long long p = (long long)r * S.cols + c;
    const double a = S.dsm[p];
    const double wall = S.walls[p];
    const uint8_t fl = S.flags[p];
    const ShadowResult s =
        shadow_walk_geo(GeoF64{S.dsm, S.vegdem, S.vegdem2}, S.rows, S.cols, r, c, a, S.vegdem[p], (fl & 2) != 0,
                        wall, reinterpret_cast<const int2*>(h.ray_dxdy), h.ray_dz, h.steps, S.hmax, true);
    // Wall planes of shadowingfunction_wallheight_23 (only the sunlit-wall
    // test of the GVF reads them); see quad_from_walk for the no-division test.
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
    const bool sunwall = (fl & 1) && wall > 0.0 && wallsun == wall;
    const double sh = s.shadowed ? 0.0 : 1.0;
    const double vegsh = s.veg ? 0.0 : 1.0;
    const double shadow = sh - (1.0 - vegsh) * (1.0 - h.psi);
    double tg = ground_tg(S, h, p);
    const double emis = S.emis[p];
    sc[kS64LupFirst * n + p] = lup_excess(emis, tg, shadow, h.ta);
    if (S.has_water && (fl & 4)) tg = h.twater - h.ta;
    sc[kS64Shadow * n + p] = shadow;
    sc[kS64Lup * n + p] = lup_excess(emis, tg, shadow, h.ta);
    sc[kS64AlbSh * n + p] = (double)S.alb[p] * shadow;
    sc[kS64Bits * n + p] = (double)((fl & 1 ? 1 : 0) | (sunwall ? 2 : 0));
}

// Ground view factors of one daytime hour into the 15 scratch GVF planes
// (the step reads no gvfSum / gvfNorm, so the shadow sums are not kept).
// Per direction the walk keeps the reference's running sums step by step
// (no closed-form remainder), so the sums are added in the same order.
__global__ void __launch_bounds__(kStep64BX* kStep64BY) step64_gvf_kernel(
    SolweigScene S, const SolweigHour* __restrict__ hours, int hour, GvfOffsets64 tab, int first, int second,
    double* __restrict__ sc) {
    const SolweigHour& h = hours[hour];
    if (!h.daytime) return;
    const int c = blockIdx.x * kStep64BX + threadIdx.x;
    const int r = blockIdx.y * kStep64BY + threadIdx.y;
    if (r >= S.rows || c >= S.cols) return;
    const long long n = (long long)S.rows * S.cols;
    const long long p = (long long)r * S.cols + c;
    const double* shp = sc + kS64Shadow * n;
    const double* lupp = sc + kS64Lup * n;
    const double* lup1p = S.has_water ? sc + kS64LupFirst * n : lupp;
    const double* albshp = sc + kS64AlbSh * n;
    const double* bitsp = sc + kS64Bits * n;
    const double ta = h.ta;
    constexpr double ewall = 0.9, albedo_b = 0.2;
    const double lwall = kSBC * ewall * pow4(h.tgwall + ta + 273.15) - kSBC * ewall * pow4(ta + 273.15);
    const double own_b = ((int)bitsp[p] & 1) ? 1.0 : 0.0;
    const double ground = 1.0 - own_b;
    const double own_sh = shp[p], own_lup = lupp[p], own_alb = (double)S.alb[p];
    const uint32_t face = S.gvf_face[p];
    const double dfirst = first, dsecond = second;
    double lup[5] = {0, 0, 0, 0, 0}, alb[5] = {0, 0, 0, 0, 0}, nosh[5] = {0, 0, 0, 0, 0};
    for (int j = 0; j < SOLWEIG_GVF_DIRECTIONS; ++j) {
        const int2* o = tab.offs + j * second;
        const double* lsrc = j == 0 ? lup1p : lupp;
        double f = own_b;
        double t_bu = 0.0, t_lup = 0.0, t_albsh = 0.0, t_alb = 0.0, t_sun = 0.0;
        double s_lup = 0.0, s_albsh = 0.0, s_alb = 0.0;
        double s_wall = 0.0, s_lwall = 0.0, s_albwall = 0.0, s_albwall_nosh = 0.0;
        double seen_sun = 0.0, seen_wall = 0.0;
        double n_wall = 0.0, n_lwall = 0.0, n_lup = 0.0, n_albwall = 0.0, n_albsh = 0.0, n_albwall_nosh = 0.0,
               n_alb = 0.0;
        for (int k = 0; k < second; ++k) {
            const int rr = r + o[k].x, cc = c + o[k].y;
            // A sample outside the raster keeps the last one seen (the
            // reference's shifted copies are not cleared between steps).
            if (in_raster(rr, cc, S.rows, S.cols)) {
                const long long q = (long long)rr * S.cols + cc;
                const int bits = (int)__ldg(&bitsp[q]);
                t_bu = (bits & 1) ? 1.0 : 0.0;
                t_sun = (bits & 2) ? 1.0 : 0.0;
                t_lup = __ldg(&lsrc[q]);
                t_albsh = __ldg(&albshp[q]);
                t_alb = (double)__ldg(&S.alb[q]);
            }
            f = fmin(f, t_bu);
            s_lup += t_lup * f;
            s_albsh += t_albsh * f;
            s_alb += t_alb * f;
            seen_sun = (t_sun * f + seen_sun) > 0.0 ? 1.0 : 0.0;
            seen_wall = ((1.0 - f) + seen_wall) > 0.0 ? 1.0 : 0.0;
            s_lwall += seen_sun * lwall;
            s_albwall += seen_sun * albedo_b;
            s_wall += seen_sun;
            s_albwall_nosh += seen_wall * albedo_b;
            if (k + 1 <= first) {
                n_wall = s_wall; n_lwall = s_lwall; n_lup = s_lup;
                n_albwall = s_albwall; n_albsh = s_albsh; n_albwall_nosh = s_albwall_nosh; n_alb = s_alb;
            }
        }
        const bool sun_near = n_wall > 0.0, wall_near = n_albwall_nosh > 0.0;
        const bool sun_far = s_wall > 0.0, wall_far = s_albwall_nosh > 0.0;
        // keep == 1 of the reference: every step saw a sunlit wall and the
        // wall face is turned away from this direction.
        if (s_wall == dsecond && ((face >> j) & 1u)) {
            s_lwall = 0.0;
            s_albwall = 0.0;
        }
        const double lup1 = sun_near ? (n_lwall + n_lup) / (dfirst + 1.0) : n_lup / dfirst;
        const double lup2 = sun_far ? (s_lwall + s_lup) / (dsecond + 1.0) : s_lup / dsecond;
        const double alb1 = sun_near ? (n_albwall + n_albsh) / (dfirst + 1.0) : n_albsh / dfirst;
        const double alb2 = sun_far ? (s_albwall + s_albsh) / (dsecond + 1.0) : s_albsh / dsecond;
        const double nosh1 = wall_near ? (n_albwall_nosh + n_alb) / (dfirst + 1.0) : n_alb / dfirst;
        const double nosh2 = wall_far ? (s_albwall_nosh + s_alb) / dsecond : s_alb / dsecond;
        const double d_lup = (lup1 * 0.5 + lup2 * 0.4) / 0.9 + own_lup * ground;
        const double d_alb = (alb1 * 0.5 + alb2 * 0.4) / 0.9 + own_alb * ground * own_sh;
        const double d_nosh = ((nosh1 * 0.5 + nosh2 * 0.4) / 0.9) * own_b + own_alb * ground;
        const unsigned groups = gvf_direction_groups(j);
#pragma unroll
        for (int g = 0; g < 5; ++g)
            if (groups & (1u << g)) {
                lup[g] += d_lup;
                alb[g] += d_alb;
                nosh[g] += d_nosh;
            }
    }
    const double ambient = kSBC * (double)S.emis[p] * pow4(ta + 273.15);
    double* gvf = sc + kS64Gvf * n;
#pragma unroll
    for (int g = 0; g < 5; ++g) {
        const double div = g == 0 ? 18.0 : 9.0;
        gvf[(long long)g * n + p] = lup[g] / div + ambient;
        gvf[(long long)(5 + g) * n + p] = alb[g] / div;
        gvf[(long long)(10 + g) * n + p] = nosh[g] / div;
    }
}

// Per-patch values of one hour (float64), staged in shared memory.
struct PatchSmem64 {
    double omega[SOLWEIG_MAX_PATCHES], ca[SOLWEIG_MAX_PATCHES], sa[SOLWEIG_MAX_PATCHES];
    double lum[SOLWEIG_MAX_PATCHES];      // Perez luminance (diffuse sum)
    double lum_chi[SOLWEIG_MAX_PATCHES];  // lum * radD / rad_tot (side diffuse)
    double x_off[SOLWEIG_MAX_PATCHES], lo[SOLWEIG_MAX_PATCHES], hi[SOLWEIG_MAX_PATCHES];
    double sky_down[SOLWEIG_MAX_PATCHES], sky_side[SOLWEIG_MAX_PATCHES];
    double card[4][SOLWEIG_MAX_PATCHES];
    uint8_t lw_test[SOLWEIG_MAX_PATCHES];
};

__device__ __forceinline__ double* state64_plane(const SolweigState64& st, int d) {
    return d == 0 ? st.tgmap1 : d == 1 ? st.tgmap1e : d == 2 ? st.tgmap1s : d == 3 ? st.tgmap1w : st.tgmap1n;
}

__device__ __forceinline__ double* kside64_plane(const SolweigOutputs64& o, int d) {
    return d == 1 ? o.keast : d == 2 ? o.ksouth : d == 3 ? o.kwest : o.knorth;
}

__device__ __forceinline__ double* lcard64_plane(const SolweigOutputs64& o, int d) {
    return d == 1 ? o.least : d == 2 ? o.lsouth : d == 3 ? o.lwest : o.lnorth;
}

// TsWaveDelay_2015a (src/umep_solweig.py:1633-1652) of one pixel: returns the
// delayed value and writes the carried state.
__device__ __forceinline__ double wave_delay64(const SolweigHour& h, double current, double* state, long long p) {
    const double prev = h.firstdaytime ? current : state[p];
    const double w = h.wave_weight;
    const double out = current * (1.0 - w) + prev * w;
    state[p] = h.wave_update ? out : prev;
    return out;
}

__device__ __forceinline__ void stage_patches64(PatchSmem64& sm, const SolweigSkyLayout& L, const SolweigSky64& K,
                                                const SolweigHour& h, const SolweigHour64& h64) {
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    const int nt = blockDim.x * blockDim.y;
    for (int k = tid; k < SOLWEIG_MAX_PATCHES; k += nt) {
        const bool ok = k < L.patches;
        const bool lit = ok && h.daytime;
        const int b = ok ? L.band_of_patch[k] : 0;
        sm.omega[k] = ok ? K.omega[k] : 0.0;
        sm.ca[k] = ok ? K.cos_alt[k] : 0.0;
        sm.sa[k] = ok ? K.sin_alt[k] : 0.0;
        sm.lum[k] = lit ? h64.lum[k] : 0.0;
        sm.lum_chi[k] = lit ? (h64.lum[k] * h.rad_d) / h.rad_tot : 0.0;
        sm.x_off[k] = ok ? h.yi[k] : 0.0;
        sm.lo[k] = ok ? L.sunlit_below[k] : 0.0;
        sm.hi[k] = ok ? L.shaded_above[k] : 0.0;
        sm.lw_test[k] = ok ? h.lw_sun_test[k] : 0;
        sm.sky_down[k] = ok ? (h64.band_lsky[b] * K.omega[k]) * K.sin_alt[k] : 0.0;
        sm.sky_side[k] = ok ? (h64.band_lsky[b] * K.omega[k]) * K.cos_alt[k] : 0.0;
        for (int d = 0; d < 4; ++d) sm.card[d][k] = ok ? K.cardinal[d][k] : 0.0;
    }
}

// One pixel-hour of the radiation epilogue in float64.  Expressions follow
// the grouping of Kup_veg_2015a, Kside_veg_v2022a, Lcyl_v2022a and the Tmrt
// expression; a 0/1 mask factor of the reference is a branch here (x * 1 is
// x and adding the x * 0 = 0 term leaves a sum unchanged).
__global__ void __launch_bounds__(kStep64BX* kStep64BY) step64_radiation_kernel(
    SolweigScene S, const double* __restrict__ svfbuveg, const SolweigSkyLayout* __restrict__ Lp,
    const SolweigSky64* __restrict__ Kp, const SolweigHour* __restrict__ hours,
    const SolweigHour64* __restrict__ hours64, int hour, SolweigState64 st, SolweigOutputs64 out,
    const double* __restrict__ sc) {
    const SolweigHour& h = hours[hour];
    const SolweigSkyLayout& L = *Lp;
    __shared__ PatchSmem64 sm;
    stage_patches64(sm, L, *Kp, h, hours64[hour]);
    __syncthreads();
    const int c = blockIdx.x * kStep64BX + threadIdx.x;
    const int r = blockIdx.y * kStep64BY + threadIdx.y;
    if (r >= S.rows || c >= S.cols) return;
    const long long n = (long long)S.rows * S.cols;
    const long long p = (long long)r * S.cols + c;
    const bool day = h.daytime != 0;
    const uint8_t fl = S.flags[p];
    const double ta = h.ta;
    const double emis = S.emis[p];
    constexpr double ewall = 0.9, albedo_b = 0.2;
    constexpr double absK = 0.7, absL = 0.95, Fside = 0.22, Fup = 0.06, Fcyl = 0.28;
    uint32_t Sw[SOLWEIG_MASK_WORDS], Vw[SOLWEIG_MASK_WORDS];
#pragma unroll
    for (int w = 0; w < SOLWEIG_MASK_WORDS; ++w) {
        Sw[w] = S.masks[(long long)w * n + p];
        Vw[w] = S.masks[(long long)(SOLWEIG_MASK_WORDS + w) * n + p];
    }
    const double tan_asvf = S.tan_asvf[p];
    const int P = L.patches;

    double shadow = 0.0, tg = 0.0, tg_out = ta;
    double kup[5] = {0, 0, 0, 0, 0}, lup[5];
    double kdown = 0.0, kside_i = 0.0, kside_d = 0.0, kside = 0.0, d_rad = 0.0;
    if (day) {
        shadow = sc[kS64Shadow * n + p];
        const double fsh = wedge_fsh(S.svfalfa[p], h.tan_zen);
        const double svb = svfbuveg[p];
        const double reflected = albedo_b * (1.0 - svb) * (h.rad_g * (1.0 - fsh) + h.rad_d * fsh);
        const double base = h.rad_d * svb + reflected;
        const double* gvf = sc + kS64Gvf * n;
#pragma unroll
        for (int d = 0; d < 5; ++d) {
            kup[d] = gvf[(long long)(5 + d) * n + p] * h.rad_i * h.sin_alt + base * gvf[(long long)(10 + d) * n + p];
            lup[d] = wave_delay64(h, gvf[(long long)d * n + p], state64_plane(st, d), p);
        }
        tg = ground_tg(S, h, p);
        if (S.has_water && (fl & 4)) tg = h.twater - ta;
        tg_out = wave_delay64(h, tg * shadow + ta, st.tgout1, p);
        // Diffuse sky: diffsh is 1 for sky patches, the float32 value of
        // 1 - (1 - transmissivity) for vegetation, 0 behind buildings.
        const double dveg = Kp->diffsh_veg;
        double lum = 0.0;
        for (int k = 0; k < P; ++k) {
            const uint32_t bit = 1u << (k & 31);
            const bool s = Sw[k >> 5] & bit, v = Vw[k >> 5] & bit;
            lum += (s ? (v ? dveg : 1.0) : 0.0) * sm.lum[k];
        }
        d_rad = lum * h.rad_d;
        kdown = h.rad_i * shadow * h.sin_alt + d_rad + reflected;
        kside_i = shadow * h.rad_i * h.cos_alt;
        const double sun_surf = (albedo_b * (h.rad_i * h.cos_alt) + (h.rad_d * 0.5)) / kPi;
        const double shade_surf = (albedo_b * h.rad_d * 0.5) / kPi;
        double ref_sun = 0.0, ref_sh = 0.0, ref_veg = 0.0;
        for (int k = 0; k < P; ++k) {
            const uint32_t bit = 1u << (k & 31);
            const bool s = Sw[k >> 5] & bit, v = Vw[k >> 5] & bit;
            const double ca = sm.ca[k], om = sm.omega[k];
            if (v) ref_veg += shade_surf * om * ca;
            kside_d += (s ? (v ? dveg : 1.0) : 0.0) * sm.lum_chi[k] * ca * om;
            if (!s && !v) {
                const double x = tan_asvf + sm.x_off[k];
                if (x < sm.lo[k]) ref_sun += sun_surf * om * ca;
                if (x > sm.hi[k]) ref_sh += shade_surf * om * ca;
            }
        }
        kside = kside_i + kside_d + ref_sun + ref_sh + ref_veg;
    } else {
        double l = kSBC * emis * pow4(0.0 + ta + 0.0 + 273.15);
        if (S.landcover == 1 && (fl & 4)) l = kSBC * 0.98 * pow4(h.twater + 273.15);
#pragma unroll
        for (int d = 0; d < 5; ++d) lup[d] = l;
    }

    // Anisotropic longwave (Lcyl_v2022a with define_patch_characteristics).
    const double tk4 = pow4(ta + 273.15);
    const double veg_surf = (ewall * kSBC * tk4) / kPi;
    const double sun_surf = (ewall * kSBC * pow4(ta + h.tgwall + 273.15)) / kPi;
    const double shade_surf = veg_surf;
    double d_sky = 0.0, d_veg = 0.0, d_sun = 0.0, d_sh = 0.0, d_ref = 0.0;
    double s_sky = 0.0, s_veg = 0.0, s_sun = 0.0, s_sh = 0.0, s_ref = 0.0;
    double card[4] = {0, 0, 0, 0};
    for (int k = 0; k < P; ++k) {
        const uint32_t bit = 1u << (k & 31);
        const bool s = Sw[k >> 5] & bit, v = Vw[k >> 5] & bit;
        const double ca = sm.ca[k], sa = sm.sa[k], om = sm.omega[k];
        if (s && !v) {
            d_sky += sm.sky_down[k];
            s_sky += sm.sky_side[k];
#pragma unroll
            for (int d = 0; d < 4; ++d) card[d] += sm.sky_side[k] * sm.card[d][k];
        }
        if (v) {
            s_veg += veg_surf * om * ca;
            d_veg += veg_surf * om * sa;
#pragma unroll
            for (int d = 0; d < 4; ++d) card[d] += veg_surf * om * ca * sm.card[d][k];
        }
        if (!s && !v) {
            if (sm.lw_test[k]) {
                const double x = tan_asvf + sm.x_off[k];
                const bool sunlit = x < sm.lo[k], shaded = x > sm.hi[k];
                if (sunlit) {
                    s_sun += sun_surf * om * ca;
                    d_sun += sun_surf * om * sa;
                }
                if (shaded) {
                    s_sh += shade_surf * om * ca;
                    d_sh += shade_surf * om * sa;
                }
#pragma unroll
                for (int d = 0; d < 4; ++d) {
                    if (sunlit) card[d] += sun_surf * om * ca * sm.card[d][k];
                    if (shaded) card[d] += shade_surf * om * ca * sm.card[d][k];
                }
            } else {
                s_sh += shade_surf * om * ca;
                d_sh += shade_surf * om * sa;
#pragma unroll
                for (int d = 0; d < 4; ++d) card[d] += shade_surf * om * ca * sm.card[d][k];
            }
        }
    }
    const double refl = ((d_sky + lup[0]) * (1.0 - ewall) * 0.5) / kPi;
    for (int k = 0; k < P; ++k) {
        const uint32_t bit = 1u << (k & 31);
        if ((Sw[k >> 5] & bit) && !(Vw[k >> 5] & bit)) continue;  // sky: not obstructed
        const double ca = sm.ca[k], om = sm.omega[k];
        s_ref += refl * om * ca;
        d_ref += refl * om * sm.sa[k];
#pragma unroll
        for (int d = 0; d < 4; ++d) card[d] += refl * om * ca * sm.card[d][k];
    }
    const double lside = s_sky + s_veg + s_sh + s_sun + s_ref;
    const double ldown = d_sky + d_veg + d_sh + d_sun + d_ref;

    // Tmrt, cylinder with anisotropic sky: Keast.. = KupE..*0.5 and
    // Least.. = LupE..*0.5 enter the sums before the patch terms are added.
    const double ksum = kup[4] * 0.5 + kup[1] * 0.5 + kup[2] * 0.5 + kup[3] * 0.5;
    const double lsum = lup[4] * 0.5 + lup[1] * 0.5 + lup[2] * 0.5 + lup[3] * 0.5;
    const double sstr = absK * (kside * Fcyl + (kdown + kup[0]) * Fup + ksum * Fside) +
                        absL * ((ldown + lup[0]) * Fup + lside * Fcyl + lsum * Fside);
    const double tmrt = sqrt(sqrt(sstr / (absL * kSBC))) - 273.2;
    if (out.tmrt) out.tmrt[p] = tmrt;
    if (out.utci)
        out.utci[p] = (fl & 1) ? utci_eval(h.utci, (double)(float)tmrt, (double)(float)ta, h.utci_valid)
                               : __int_as_float(0x7fc00000);
    if (out.kdown) out.kdown[p] = kdown;
    if (out.kup) out.kup[p] = kup[0];
    if (out.ldown) out.ldown[p] = ldown;
    if (out.lup) out.lup[p] = lup[0];
    if (out.shadow) out.shadow[p] = shadow;
    if (out.tg) out.tg[p] = tg;
    // Cardinal planes: E, S, W, N = direction 1..4 of the GVF; the longwave
    // patch terms are accumulated as E, S, W, N (card[0..3]).
#pragma unroll
    for (int d = 1; d < 5; ++d) {
        double* ko = kside64_plane(out, d);
        if (ko) ko[p] = kup[d] * 0.5;
        double* lo = lcard64_plane(out, d);
        if (lo) lo[p] = lup[d] * 0.5 + card[d - 1];
    }
    if (out.kside_i) out.kside_i[p] = kside_i;
    if (out.kside_d) out.kside_d[p] = kside_d;
    if (out.kside) out.kside[p] = kside;
    if (out.lside) out.lside[p] = lside;
    if (out.d_rad) out.d_rad[p] = d_rad;
    if (out.tg_out) out.tg_out[p] = tg_out;
}

}  // namespace solweig

using namespace solweig;

extern "C" int solweig_step64(const SolweigScene* scene, const double* svfbuveg, const SolweigSkyLayout* layout,
                              const SolweigSky64* sky, const SolweigHour* hours, const SolweigHour64* hours64,
                              int hour, const SolweigState64* state, const SolweigOutputs64* out,
                              const int32_t* gvf_dxdy, int first_steps, int second_steps, double* scratch,
                              void* stream) {
    SOLWEIG_CHECK_ARG(scene && svfbuveg && layout && sky && hours && hours64 && hour >= 0 && state && out &&
                          gvf_dxdy && scratch,
                      "solweig_step64: null argument");
    const SolweigScene& S = *scene;
    SOLWEIG_CHECK_ARG(S.rows > 0 && S.cols > 0 && S.rows < (1 << 20) && S.cols < (1 << 20),
                      "solweig_step64: bad scene shape %dx%d", S.rows, S.cols);
    SOLWEIG_CHECK_ARG(S.dsm && S.vegdem && S.vegdem2 && S.walls && S.aspect && S.flags && S.alb && S.emis &&
                          S.tgk && S.tstart && S.tmaxlst && S.svfalfa && S.tan_asvf && S.masks && S.gvf_face,
                      "solweig_step64: scene has a null array");
    SOLWEIG_CHECK_ARG(state->tgmap1 && state->tgmap1e && state->tgmap1s && state->tgmap1w && state->tgmap1n &&
                          state->tgout1,
                      "solweig_step64: state has a null plane");
    SOLWEIG_CHECK_ARG(second_steps >= 1 && second_steps <= SOLWEIG_GVF_MAX_STEPS && first_steps >= 1 &&
                          first_steps <= second_steps,
                      "solweig_step64: GVF steps first=%d second=%d", first_steps, second_steps);
    GvfOffsets64 tab;
    for (int i = 0; i < SOLWEIG_GVF_DIRECTIONS * second_steps; ++i)
        tab.offs[i] = make_int2(gvf_dxdy[2 * i], gvf_dxdy[2 * i + 1]);
    cudaStream_t st = as_stream(stream);
    dim3 block(kStep64BX, kStep64BY);
    dim3 grid(blocks_for(S.cols, kStep64BX), blocks_for(S.rows, kStep64BY));
    step64_fields_kernel<<<grid, block, 0, st>>>(S, hours, hour, scratch);
    SOLWEIG_CHECK_LAUNCH("step64_fields_kernel");
    step64_gvf_kernel<<<grid, block, 0, st>>>(S, hours, hour, tab, first_steps, second_steps, scratch);
    SOLWEIG_CHECK_LAUNCH("step64_gvf_kernel");
    step64_radiation_kernel<<<grid, block, 0, st>>>(S, svfbuveg, layout, sky, hours, hours64, hour, *state, *out,
                                                    scratch);
    SOLWEIG_CHECK_LAUNCH("step64_radiation_kernel");
    return SOLWEIG_OK;
}
