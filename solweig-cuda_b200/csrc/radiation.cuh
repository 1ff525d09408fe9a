// Per-pixel radiation epilogue of one hour: patch sums, fluxes, Tmrt, UTCI.
//
// Restates the cyl = 1, anisotropic-sky path of Solweig_2022a_calc
// (src/umep_solweig.py:50-372) with Kside_veg_v2022a (:666-911),
// Lcyl_v2022a / define_patch_characteristics (:946-1028, :1205-1356),
// Kup_veg_2015a (:915-927), TsWaveDelay_2015a (:1633-1652),
// cylindric_wedge (:383-426) and the Tmrt expression (:345-360); the UTCI
// polynomial of src/kernels/utci.cu evaluated in (Tmrt - Ta) with the seven
// hourly coefficients computed on the host.
//
// Patch sums use the packed visibility words.  Within one altitude band the
// solid angle and cos/sin of the altitude are the same for every patch, so
// every static sum is a per-band popcount (computed once after the SVF); only
// the Perez luminance weights (sky / vegetation patches) and the sunlit/shaded
// split of building patches change every hour.
#pragma once
#include "common.cuh"

namespace solweig {

// Per-patch values of one hour staged in shared memory (divergent indexing).
struct PatchSmem {
    float lum[SOLWEIG_MAX_PATCHES];      // Perez luminance
    float lum_cw[SOLWEIG_MAX_PATCHES];   // luminance * cos(alt) * omega
    float wcos[SOLWEIG_MAX_PATCHES];     // omega * cos(alt)
    float wsin[SOLWEIG_MAX_PATCHES];     // omega * sin(alt)
    double x_off[SOLWEIG_MAX_PATCHES];   // yi (added to tan(asvf))
    double lo[SOLWEIG_MAX_PATCHES];      // sunlit below
    double hi[SOLWEIG_MAX_PATCHES];      // shaded above
    uint8_t lw_test[SOLWEIG_MAX_PATCHES];
    float card[4][SOLWEIG_MAX_PATCHES];  // longwave E,S,W,N cosines (0 = not in that half)
    float lsky_side[SOLWEIG_MAX_PATCHES];  // sky longwave of the patch on a vertical surface
    float band_down[SOLWEIG_MAX_BANDS];  // sky longwave per visible patch, horizontal
    float band_side[SOLWEIG_MAX_BANDS];  // sky longwave per visible patch, vertical
    uint32_t valid[SOLWEIG_MASK_WORDS];  // bits of existing patches
};

__device__ __forceinline__ void stage_patches(PatchSmem& sm, const SolweigSkyLayout& L,
                                              const SolweigHour& h) {
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    const int nt = blockDim.x * blockDim.y;
    for (int k = tid; k < SOLWEIG_MAX_PATCHES; k += nt) {
        const bool ok = k < L.patches;
        sm.lum[k] = ok ? h.lum[k] : 0.f;
        sm.lum_cw[k] = ok ? h.lum[k] * L.cos_alt[k] * L.omega[k] : 0.f;
        sm.wcos[k] = ok ? L.omega[k] * L.cos_alt[k] : 0.f;
        sm.wsin[k] = ok ? L.omega[k] * L.sin_alt[k] : 0.f;
        sm.x_off[k] = ok ? h.yi[k] : 0.0;
        sm.lo[k] = ok ? L.sunlit_below[k] : 0.0;
        sm.hi[k] = ok ? L.shaded_above[k] : 0.0;
        sm.lw_test[k] = ok ? h.lw_sun_test[k] : 0;
        for (int d = 0; d < 4; ++d) sm.card[d][k] = ok ? L.cardinal[d][k] : 0.f;
        const int b = ok ? L.band_of_patch[k] : 0;
        sm.lsky_side[k] = ok ? h.band_lsky[b] * L.band_omega[b] * L.band_cos[b] : 0.f;
    }
    if (tid < SOLWEIG_MAX_BANDS) {
        const bool ok = tid < L.nbands;
        sm.band_down[tid] = ok ? h.band_lsky[tid] * L.band_omega[tid] * L.band_sin[tid] : 0.f;
        sm.band_side[tid] = ok ? h.band_lsky[tid] * L.band_omega[tid] * L.band_cos[tid] : 0.f;
    }
    if (tid < SOLWEIG_MASK_WORDS) {
        const int lo = tid * 32;
        const int nbits = L.patches - lo;
        sm.valid[tid] = nbits >= 32 ? 0xffffffffu : (nbits <= 0 ? 0u : ((1u << nbits) - 1u));
    }
}

// Results of the per-pixel patch loop (weights, before hour scaling).
struct PatchSums {
    float lum_sky, lum_veg;        // sum of luminance over sky / vegetation patches
    float cw_sky, cw_veg;          // same, times cos(alt)*omega
    float sw_sun, sw_shade;        // omega*cos over building patches sunlit / shaded (shortwave)
    float lw_sun_c, lw_shade_c;    // omega*cos, building patches sunlit / shaded (longwave)
    float lw_sun_s, lw_shade_s;    // omega*sin, same
    float card_sky[4], card_veg[4], card_sun[4], card_shade[4], card_obst[4];
};

template <bool Cardinal>
__device__ __forceinline__ PatchSums patch_loop(const PatchSmem& sm, const uint32_t* S,
                                                const uint32_t* V, double tan_asvf, bool daytime) {
    PatchSums ps{};
#pragma unroll
    for (int w = 0; w < SOLWEIG_MASK_WORDS; ++w) {
        const uint32_t valid = sm.valid[w];
        const uint32_t sky = S[w] & ~V[w] & valid;
        const uint32_t veg = S[w] & V[w] & valid;
        const uint32_t bld = ~S[w] & ~V[w] & valid;
        if (daytime) {
            for (uint32_t m = sky; m; m &= m - 1) {
                const int k = w * 32 + __ffs(m) - 1;
                ps.lum_sky += sm.lum[k];
                ps.cw_sky += sm.lum_cw[k];
            }
            for (uint32_t m = veg; m; m &= m - 1) {
                const int k = w * 32 + __ffs(m) - 1;
                ps.lum_veg += sm.lum[k];
                ps.cw_veg += sm.lum_cw[k];
            }
        }
        for (uint32_t m = bld; m; m &= m - 1) {
            const int k = w * 32 + __ffs(m) - 1;
            const double x = tan_asvf + sm.x_off[k];
            const bool sunlit = x < sm.lo[k];
            const bool shaded = x > sm.hi[k];
            if (daytime) {
                if (sunlit) ps.sw_sun += sm.wcos[k];
                if (shaded) ps.sw_shade += sm.wcos[k];
            }
            const bool test = sm.lw_test[k] != 0;
            const bool lsun = test && sunlit;
            const bool lshade = !test || shaded;
            if (lsun) {
                ps.lw_sun_c += sm.wcos[k];
                ps.lw_sun_s += sm.wsin[k];
            }
            if (lshade) {
                ps.lw_shade_c += sm.wcos[k];
                ps.lw_shade_s += sm.wsin[k];
            }
            if (Cardinal) {
#pragma unroll
                for (int d = 0; d < 4; ++d) {
                    if (lsun) ps.card_sun[d] += sm.wcos[k] * sm.card[d][k];
                    if (lshade) ps.card_shade[d] += sm.wcos[k] * sm.card[d][k];
                }
            }
        }
        if (Cardinal) {
            for (uint32_t m = sky; m; m &= m - 1) {
                const int k = w * 32 + __ffs(m) - 1;
#pragma unroll
                for (int d = 0; d < 4; ++d) ps.card_sky[d] += sm.lsky_side[k] * sm.card[d][k];
            }
            const uint32_t vmask = V[w] & valid;
            for (uint32_t m = vmask; m; m &= m - 1) {
                const int k = w * 32 + __ffs(m) - 1;
#pragma unroll
                for (int d = 0; d < 4; ++d) ps.card_veg[d] += sm.wcos[k] * sm.card[d][k];
            }
            const uint32_t obst = ~(S[w] & ~V[w]) & valid;
            for (uint32_t m = obst; m; m &= m - 1) {
                const int k = w * 32 + __ffs(m) - 1;
#pragma unroll
                for (int d = 0; d < 4; ++d) ps.card_obst[d] += sm.wcos[k] * sm.card[d][k];
            }
        }
    }
    return ps;
}

// UTCI from the hour's collapsed polynomial in D = Tmrt - Ta.
__device__ __forceinline__ float utci_eval(const double* c, double tmrt, double ta, int valid) {
    if (!valid || tmrt <= -999.0) return -999.0f;
    const double d = tmrt - ta;
    double u = c[6];
#pragma unroll
    for (int i = 5; i >= 0; --i) u = u * d + c[i];
    return (float)u;
}

// Fraction of shaded wall, cylindric_wedge (NaN -> 0.5), from ta = tan(svfalfa).
__device__ __forceinline__ double wedge_fsh_tan(double ta, double tan_zen) {
    const double xa = 1.0 - 2.0 / (ta * tan_zen);
    const double ha = 2.0 / (ta * tan_zen);
    const double ba = 1.0 / ta;
    const double hkil = 2.0 * ba * ha;
    double ukil = 0.0;
    if (xa < 0.0) {
        const double qa = tan_zen / 2.0;
        const double za = sqrt(ba * ba - qa * qa / 4.0);
        const double phi = atan(za / qa);
        const double area = (sin(phi) - phi * cos(phi)) / (1.0 - cos(phi));
        ukil = 2.0 * ba * xa * area;
    }
    const double fsh = (2.0 * kPi * ba - (hkil + ukil)) / (2.0 * kPi * ba);
    return isnan(fsh) ? 0.5 : fsh;
}

__device__ __forceinline__ double wedge_fsh(double svfalfa, double tan_zen) {
    return wedge_fsh_tan(tan(svfalfa), tan_zen);
}

}  // namespace solweig
