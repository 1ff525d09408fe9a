// Gradient of a day's mean UTCI (or Tmrt) with the shadow and SVF masks held
// fixed: a hand-written reverse pass of the batched day.
//
// Parameters (per pixel): ground albedo a, ground emissivity e and the
// direct-beam transmissivity t of vegetation, which replaces the hour's psi
// in shadow = sh - (1 - vegsh)(1 - t) (src/umep_solweig.py:171 of the step;
// the diffuse-sky transmissivity 0.03 of the SVF stays fixed).  Forcing: the
// kernels return the partials of the objective with respect to the per-hour
// scalars the device consumes (Ta, direct and diffuse radiation, their
// normaliser, CI_TgG, the wall temperature, the 8 band sky emittances, the 7
// UTCI coefficients and, through the contraction, the Perez luminances);
// the host chains them with the Jacobian of its FP64 hour plan.
//
//  forward (also re-run by the backward: per-hour recomputation, nothing is
//  kept from the forward call)
//    day_shadow_kernel        masks of every hour (shadow sweep, psi of the hour)
//    param_quads_kernel       GVF field quads from the parameters: shadow with t,
//                             Lup with e, albedo a
//    day_gvf_kernel           all-direction GVF of every hour (scene copy with e, a)
//    contraction              luminance sums (mask-only, parameter-free)
//    grad_radiation_kernel    per pixel: forward over the hours (states kept),
//                             objective, then backward over the hours, each
//                             hour's fluxes recomputed from its inputs
//  backward
//    gvf_adjoint_kernel       transpose of the GVF walk: scatter the adjoints of
//                             the GVF planes onto the walked pixels' Lup,
//                             albedo*shadow and albedo (atomics)
//    param_grad_kernel        per pixel: chain to a, e, t; Ta / CI_TgG partials
//    lum_grad_kernel          mask-transpose sums for the Perez luminances
#include "day_kernels.cuh"

namespace solweig {
namespace {

enum HourField {
    kGTa = 0,
    kGRadI,
    kGRadD,
    kGRadTot,
    kGCiTgg,
    kGTgwall,
    kGBand0,                   // 8 band sky emittances
    kGUtci0 = kGBand0 + 8,     // 7 UTCI coefficients
    kGFields = kGUtci0 + 7
};
static_assert(kGFields == SOLWEIG_GRAD_HOUR_FIELDS, "hour field count");

constexpr double kEwall = 0.9, kAlbB = 0.2;
constexpr double kAbsK = 0.7, kAbsL = 0.95, kFside = 0.22, kFup = 0.06, kFcyl = 0.28;

struct GradPtrs {
    const float* alb;
    const float* emis;
    const float* tau;
    const uint8_t* sv;      // [H][px] bit0 sh (sunlit of buildings), bit1 vegsh (no canopy shade)
    const float4* quads;    // [H][px] parameter quads
    const float* gvf;       // [H][3][px]
    const float* nosh;      // [px]
    const float* sums;      // [2 * ncols][px]
    int ncols;
    // adjoint outputs of the radiation pass
    float* lam_gl;          // [H][px]
    float* lam_ga;          // [H][px]
    float* lam_gn;          // [H][px]
    float* lam_s;           // [H][px]  own shadow
    float* lam_sums;        // [H][4][px]
    float* d_emis_direct;   // [px]
    double* hour_grad;      // [H][kGFields]
    double* daily;          // [px] objective per pixel (forward)
    const float* weights;   // [px] dJ/d daily (backward), or null for forward only
    int objective;          // 0 UTCI, 1 Tmrt
};

// ------------------------------------------------------------------ quads

// Decode the building / canopy masks from the forward quads (shadow value with
// the hour's psi) and rebuild the quads with the parameters.
__global__ void param_quads_kernel(SolweigScene S, const SolweigHour* __restrict__ hours, int nhours,
                                   const float4* __restrict__ q0, float4* __restrict__ q1,
                                   uint8_t* __restrict__ sv, const float* __restrict__ alb,
                                   const float* __restrict__ emis, const float* __restrict__ tau) {
    const long long n = (long long)S.rows * S.cols;
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= n * nhours) return;
    const int hr = (int)(idx / n);
    const long long p = idx - (long long)hr * n;
    const SolweigHour& h = hours[hr];
    if (!h.daytime) return;
    const float4 q = q0[idx];
    const float s0 = q.x;
    const float psi = (float)h.psi;
    // shadow = (float)(sh - (1 - vegsh)(1 - psi)): 1, psi, 0 or psi - 1
    int sh, vegsh;
    if (s0 == 1.0f) { sh = 1; vegsh = 1; }
    else if (s0 == 0.0f) { sh = 0; vegsh = 1; }
    else if (s0 == (float)(1.0 - (1.0 - h.psi))) { sh = 1; vegsh = 0; }
    else { sh = 0; vegsh = 0; }
    (void)psi;
    sv[idx] = (uint8_t)(sh | (vegsh << 1));
    const double t = tau[p];
    const double shadow = (double)(float)((double)sh - (1.0 - vegsh) * (1.0 - t));
    const double tg = ground_tg(S, h, p);
    const float lup = (float)lup_excess((double)emis[p], tg, shadow, h.ta);
    q1[idx] = make_float4((float)shadow, lup, alb[p], q.w);
}

// ------------------------------------------------------------------ radiation

struct HourIn {
    bool day;
    double s, gl, ga;
    double Ls, Cs, Lv, Cv;
};

// Everything of one pixel-hour the reverse pass needs beyond the state.
template <int OPT>
struct PixelStatics {
    uint32_t bld[SOLWEIG_MASK_WORDS];
    uint32_t cnt_lo, cnt_hi;
    bool ground;
    double emis, svfbuveg, tan_alfa, tan_asvf, vc, vs, oc, os, gn;
    __device__ double cnt(int b) const {
        return (double)(((b < 4 ? cnt_lo : cnt_hi) >> (8 * (b & 3))) & 0xFFu);
    }
};

struct BuildingTerms {
    double sws, swh, lsu_c, lsu_s, lsh_c, lsh_s;
};

template <int OPT>
__device__ BuildingTerms building_terms(const DayTable& T, const PixelStatics<OPT>& ps, int P, const float* wcos,
                                        const float* wsin) {
    const int isun = count_le(T.tsun, P, ps.tan_asvf);
    const int ishd = count_le(T.vshade, P, ps.tan_asvf);
    uint32_t m_sun[SOLWEIG_MASK_WORDS], m_shd[SOLWEIG_MASK_WORDS], m_lsun[SOLWEIG_MASK_WORDS],
        m_lshd[SOLWEIG_MASK_WORDS];
#pragma unroll
    for (int w = 0; w < SOLWEIG_MASK_WORDS; ++w) {
        const uint32_t test = T.test[w];
        m_sun[w] = ps.bld[w] & T.suf[isun][w];
        m_shd[w] = ps.bld[w] & T.pre[ishd][w];
        m_lsun[w] = m_sun[w] & test;
        m_lshd[w] = ps.bld[w] & (~test | m_shd[w]);
    }
    BuildingTerms b;
    b.sws = band_weighted<OPT>(m_sun, wcos);
    b.swh = band_weighted<OPT>(m_shd, wcos);
    b.lsu_c = band_weighted<OPT>(m_lsun, wcos);
    b.lsu_s = band_weighted<OPT>(m_lsun, wsin);
    b.lsh_c = band_weighted<OPT>(m_lshd, wcos);
    b.lsh_s = band_weighted<OPT>(m_lshd, wsin);
    return b;
}

struct HourOut {
    double sstr, lup;
};

// Forward of one pixel-hour given the incoming state; returns sstr and Lup
// and the outgoing state.
template <int OPT>
__device__ HourOut hour_forward(const SolweigHour& h, const SolweigSkyLayout& L, const PixelStatics<OPT>& ps,
                                const HourIn& in, const BuildingTerms& bt, double state_in, double& state_out) {
    const double ta = h.ta, tk = ta + 273.15;
    double kup = 0.0, lup, kdown = 0.0, kside = 0.0;
    state_out = state_in;
    if (in.day) {
        const double fsh = wedge_fsh_tan(ps.tan_alfa, h.tan_zen);
        const double reflK = kAlbB * (1.0 - ps.svfbuveg) * (h.rad_g * (1.0 - fsh) + h.rad_d * fsh);
        const double base_up = h.rad_d * ps.svfbuveg + reflK;
        const double direct_up = h.rad_i * h.sin_alt;
        kup = in.ga * direct_up + base_up * ps.gn;
        const double prev = h.firstdaytime ? in.gl : state_in;
        lup = in.gl * (1.0 - h.wave_weight) + prev * h.wave_weight;
        state_out = h.wave_update ? lup : prev;
        const double d_rad = h.rad_d * (in.Ls + 0.03 * in.Lv);
        kdown = h.rad_i * in.s * h.sin_alt + d_rad + reflK;
        const double kside_i = in.s * h.rad_i * h.cos_alt;
        const double kside_d = (h.rad_d / h.rad_tot) * (in.Cs + 0.03 * in.Cv);
        const double sw_shade = (kAlbB * h.rad_d * 0.5) / kPi;
        const double sw_sun = (kAlbB * (h.rad_i * h.cos_alt) + h.rad_d * 0.5) / kPi;
        kside = kside_i + kside_d + sw_sun * bt.sws + sw_shade * bt.swh + sw_shade * ps.vc;
    } else {
        lup = kSBC * ps.emis * pow4(tk);
    }
    double ld_sky = 0.0, ls_sky = 0.0;
#pragma unroll
    for (int b = 0; b < 8; ++b) {
        const double bl = b < L.nbands ? (double)h.band_lsky[b] * L.band_omega[b] : 0.0;
        ld_sky += bl * L.band_sin[b] * ps.cnt(b);
        ls_sky += bl * L.band_cos[b] * ps.cnt(b);
    }
    const double lw_shade = (kEwall * kSBC * pow4(tk)) / kPi;
    const double lw_sun = in.day ? (kEwall * kSBC * pow4(ta + h.tgwall + 273.15)) / kPi : 0.0;
    const double refl = ((ld_sky + lup) * (1.0 - kEwall) * 0.5) / kPi;
    const double ldown = ld_sky + lw_shade * (ps.vs + bt.lsh_s) + lw_sun * bt.lsu_s + refl * ps.os;
    const double lside = ls_sky + lw_shade * (ps.vc + bt.lsh_c) + lw_sun * bt.lsu_c + refl * ps.oc;
    HourOut o;
    o.sstr = kAbsK * (kside * kFcyl + (kdown + kup) * kFup + 2.0 * kup * kFside) +
             kAbsL * ((ldown + lup) * kFup + lside * kFcyl + 2.0 * lup * kFside);
    o.lup = lup;
    return o;
}

// Reverse of one pixel-hour.  lam_state: adjoint of the outgoing state in,
// of the incoming state out.  Hour-scalar partials are added to acc[].
template <int OPT>
__device__ void hour_backward(const SolweigHour& h, const SolweigSkyLayout& L, const PixelStatics<OPT>& ps,
                              const HourIn& in, const BuildingTerms& bt, double state_in, double lam_obj,
                              int objective, double& lam_state, double* acc, double& d_emis, double& lam_gl,
                              double& lam_ga, double& lam_gn, double& lam_s, double* lam_sum) {
    const double ta = h.ta, tk = ta + 273.15;
    double st_out;
    const HourOut o = hour_forward<OPT>(h, L, ps, in, bt, state_in, st_out);
    const double x = o.sstr / (kAbsL * kSBC);
    const double tmrt = sqrt(sqrt(x)) - 273.2;
    double lam_tmrt = 0.0;
    if (objective == 0) {
        if (ps.ground && h.utci_valid && tmrt > -999.0) {
            const double D = tmrt - ta;
            double dpoly = 0.0, pw = 1.0;
            for (int i = 1; i <= 6; ++i) {
                dpoly += i * h.utci[i] * pw;
                pw *= D;
            }
            double pw2 = 1.0;
            for (int i = 0; i <= 6; ++i) {
                acc[kGUtci0 + i] += lam_obj * pw2;
                pw2 *= D;
            }
            lam_tmrt = lam_obj * dpoly;
            acc[kGTa] -= lam_tmrt;
        }
    } else {
        lam_tmrt = lam_obj;
    }
    const double lam_sstr = lam_tmrt * 0.25 * pow(x, -0.75) / (kAbsL * kSBC);
    const double lam_kside = kAbsK * kFcyl * lam_sstr;
    const double lam_kdown = kAbsK * kFup * lam_sstr;
    const double lam_kup = kAbsK * (kFup + 2.0 * kFside) * lam_sstr;
    const double lam_ldown = kAbsL * kFup * lam_sstr;
    const double lam_lside = kAbsL * kFcyl * lam_sstr;
    double lam_lup = kAbsL * (kFup + 2.0 * kFside) * lam_sstr;
    const double lam_refl = lam_ldown * ps.os + lam_lside * ps.oc;
    const double crefl = (1.0 - kEwall) * 0.5 / kPi;
    lam_lup += lam_refl * crefl;
    const double lam_ldsky = lam_ldown + lam_refl * crefl;
    const double lam_lssky = lam_lside;
#pragma unroll
    for (int b = 0; b < 8; ++b) {
        if (b < L.nbands)
            acc[kGBand0 + b] += ((double)L.band_omega[b]) * ps.cnt(b) *
                                (lam_ldsky * L.band_sin[b] + lam_lssky * L.band_cos[b]);
    }
    const double lam_lw_shade = lam_ldown * (ps.vs + bt.lsh_s) + lam_lside * (ps.vc + bt.lsh_c);
    acc[kGTa] += lam_lw_shade * kEwall * kSBC * 4.0 * tk * tk * tk / kPi;
    lam_gl = lam_ga = lam_gn = lam_s = 0.0;
    lam_sum[0] = lam_sum[1] = lam_sum[2] = lam_sum[3] = 0.0;
    if (in.day) {
        const double lam_lw_sun = lam_ldown * bt.lsu_s + lam_lside * bt.lsu_c;
        const double tw = ta + h.tgwall + 273.15;
        const double dlw = kEwall * kSBC * 4.0 * tw * tw * tw / kPi;
        acc[kGTa] += lam_lw_sun * dlw;
        acc[kGTgwall] += lam_lw_sun * dlw;
        // Kside
        acc[kGRadI] += lam_kside * bt.sws * kAlbB * h.cos_alt / kPi;
        acc[kGRadD] += lam_kside * (bt.sws * 0.5 / kPi + (bt.swh + ps.vc) * kAlbB * 0.5 / kPi);
        const double csum = in.Cs + 0.03 * in.Cv;
        acc[kGRadD] += lam_kside * csum / h.rad_tot;
        acc[kGRadTot] -= lam_kside * h.rad_d * csum / (h.rad_tot * h.rad_tot);
        lam_sum[1] = lam_kside * h.rad_d / h.rad_tot;
        lam_sum[3] = 0.03 * lam_kside * h.rad_d / h.rad_tot;
        lam_s += lam_kside * h.rad_i * h.cos_alt;
        acc[kGRadI] += lam_kside * in.s * h.cos_alt;
        // Kdown
        lam_s += lam_kdown * h.rad_i * h.sin_alt;
        acc[kGRadI] += lam_kdown * in.s * h.sin_alt;
        acc[kGRadD] += lam_kdown * (in.Ls + 0.03 * in.Lv);
        lam_sum[0] = lam_kdown * h.rad_d;
        lam_sum[2] = 0.03 * lam_kdown * h.rad_d;
        double lam_reflK = lam_kdown;
        // Kup
        const double fsh = wedge_fsh_tan(ps.tan_alfa, h.tan_zen);
        const double reflK = kAlbB * (1.0 - ps.svfbuveg) * (h.rad_g * (1.0 - fsh) + h.rad_d * fsh);
        const double base_up = h.rad_d * ps.svfbuveg + reflK;
        const double direct_up = h.rad_i * h.sin_alt;
        lam_ga = lam_kup * direct_up;
        lam_gn = lam_kup * base_up;
        acc[kGRadI] += lam_kup * in.ga * h.sin_alt;
        const double lam_base = lam_kup * ps.gn;
        acc[kGRadD] += lam_base * ps.svfbuveg;
        lam_reflK += lam_base;
        acc[kGRadD] += lam_reflK * kAlbB * (1.0 - ps.svfbuveg) * fsh;
        // wave delay of the GVF Lup
        const double lam_lup_total = lam_lup + (h.wave_update ? lam_state : 0.0);
        const double lam_prev = lam_lup_total * h.wave_weight + (h.wave_update ? 0.0 : lam_state);
        lam_gl = lam_lup_total * (1.0 - h.wave_weight) + (h.firstdaytime ? lam_prev : 0.0);
        lam_state = h.firstdaytime ? 0.0 : lam_prev;
        // ambient term of the GVF Lup plane: SBC * e * Tk^4
        d_emis += lam_gl * kSBC * pow4(tk);
        acc[kGTa] += lam_gl * kSBC * ps.emis * 4.0 * tk * tk * tk;
    } else {
        d_emis += lam_lup * kSBC * pow4(tk);
        acc[kGTa] += lam_lup * kSBC * ps.emis * 4.0 * tk * tk * tk;
        // the state passes through a night hour unchanged
    }
}

constexpr int kGradThreads = 128;
constexpr int kMaxGradHours = 32;

template <int OPT>
__global__ void __launch_bounds__(kGradThreads) grad_radiation_kernel(SolweigScene S, const SolweigSkyLayout* Lp,
                                                                      const SolweigHour* __restrict__ hours,
                                                                      int nhours, const DayTable* __restrict__ tables,
                                                                      GradPtrs g) {
    __shared__ float wcos[8], wsin[8];
    __shared__ double red[kGradThreads / 32][kGFields];
    const SolweigSkyLayout& L = *Lp;
    if (threadIdx.x < 8) {
        const int b = threadIdx.x;
        const int k0 = Bands<OPT>::off(b);
        wcos[b] = b < L.nbands ? L.omega[k0] * L.cos_alt[k0] : 0.f;
        wsin[b] = b < L.nbands ? L.omega[k0] * L.sin_alt[k0] : 0.f;
    }
    __syncthreads();
    const long long n = (long long)S.rows * S.cols;
    const long long p = (long long)blockIdx.x * kGradThreads + threadIdx.x;
    const bool in_range = p < n;
    const long long q = in_range ? p : 0;
    PixelStatics<OPT> ps;
#pragma unroll
    for (int w = 0; w < SOLWEIG_MASK_WORDS; ++w) {
        const int nbits = S.patches - 32 * w;
        const uint32_t valid = nbits >= 32 ? 0xffffffffu : (nbits <= 0 ? 0u : ((1u << nbits) - 1u));
        ps.bld[w] = ~S.masks[(long long)w * n + q] & ~S.masks[(long long)(SOLWEIG_MASK_WORDS + w) * n + q] & valid;
    }
    ps.cnt_lo = ps.cnt_hi = 0;
    for (int b = 0; b < 4; ++b) {
        ps.cnt_lo |= (uint32_t)S.sky_band_counts[(long long)b * n + q] << (8 * b);
        ps.cnt_hi |= (uint32_t)(b + 4 < S.nbands ? S.sky_band_counts[(long long)(b + 4) * n + q] : 0) << (8 * b);
    }
    ps.ground = (S.flags[q] & 1) != 0;
    ps.emis = g.emis[q];
    ps.svfbuveg = S.svfbuveg[q];
    ps.tan_alfa = tan(S.svfalfa[q]);
    ps.tan_asvf = S.tan_asvf[q];
    ps.vc = S.veg_sums[q];
    ps.vs = S.veg_sums[n + q];
    ps.oc = S.veg_sums[2 * n + q];
    ps.os = S.veg_sums[3 * n + q];
    ps.gn = g.nosh[q];

    auto hour_in = [&](int hr) {
        HourIn in;
        in.day = hours[hr].daytime != 0;
        in.s = in.gl = in.ga = in.Ls = in.Cs = in.Lv = in.Cv = 0.0;
        if (in.day) {
            const long long g0 = 3LL * hr * n + q;
            in.gl = g.gvf[g0];
            in.ga = g.gvf[g0 + n];
            in.s = g.gvf[g0 + 2 * n];
            const long long s0 = 2LL * hr;
            in.Ls = g.sums[s0 * n + q];
            in.Cs = g.sums[(s0 + 1) * n + q];
            in.Lv = g.sums[(g.ncols + s0) * n + q];
            in.Cv = g.sums[(g.ncols + s0 + 1) * n + q];
        }
        return in;
    };

    // forward over the hours: incoming state of every hour, objective
    double state_in[kMaxGradHours];
    double st = 0.0, obj = 0.0;
    int counted = 0;
    for (int hr = 0; hr < nhours; ++hr) {
        const SolweigHour& h = hours[hr];
        const HourIn in = hour_in(hr);
        const BuildingTerms bt = building_terms<OPT>(tables[hr], ps, S.patches, wcos, wsin);
        state_in[hr] = st;
        double st2;
        const HourOut o = hour_forward<OPT>(h, L, ps, in, bt, st, st2);
        st = st2;
        const double tmrt = sqrt(sqrt(o.sstr / (kAbsL * kSBC))) - 273.2;
        if (g.objective == 0) {
            obj += ps.ground ? (double)utci_eval(h.utci, tmrt, h.ta, h.utci_valid) : 0.0;
        } else {
            obj += tmrt;
        }
        ++counted;
    }
    const double daily = obj / (double)nhours;
    if (!g.weights) {
        if (in_range) g.daily[p] = (g.objective == 0 && !ps.ground) ? __longlong_as_double(0x7ff8000000000000ll) : daily;
        return;
    }
    // backward over the hours, each hour recomputed from its inputs
    const double w = in_range ? (double)g.weights[p] : 0.0;
    const double lam_obj = (g.objective == 0 && !ps.ground) ? 0.0 : w / (double)nhours;
    double lam_state = 0.0, d_emis = 0.0;
    for (int hr = nhours - 1; hr >= 0; --hr) {
        const SolweigHour& h = hours[hr];
        const HourIn in = hour_in(hr);
        const BuildingTerms bt = building_terms<OPT>(tables[hr], ps, S.patches, wcos, wsin);
        double acc[kGFields];
#pragma unroll
        for (int f = 0; f < kGFields; ++f) acc[f] = 0.0;
        double lgl, lga, lgn, ls, lsum[4];
        hour_backward<OPT>(h, L, ps, in, bt, state_in[hr], lam_obj, g.objective, lam_state, acc, d_emis, lgl, lga,
                           lgn, ls, lsum);
        if (in_range) {
            g.lam_gl[hr * n + p] = (float)lgl;
            g.lam_ga[hr * n + p] = (float)lga;
            g.lam_gn[hr * n + p] = (float)lgn;
            g.lam_s[hr * n + p] = (float)ls;
            for (int i = 0; i < 4; ++i) g.lam_sums[(4LL * hr + i) * n + p] = (float)lsum[i];
        }
        // block reduction of the hour-scalar partials
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
        for (int f = 0; f < kGFields; ++f) {
            double v = in_range ? acc[f] : 0.0;
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            if (lane == 0) red[warp][f] = v;
        }
        __syncthreads();
        if (threadIdx.x < kGFields) {
            double v = 0.0;
            for (int i = 0; i < kGradThreads / 32; ++i) v += red[i][threadIdx.x];
            atomicAdd(&g.hour_grad[hr * kGFields + threadIdx.x], v);
        }
        __syncthreads();
    }
    if (in_range) g.d_emis_direct[p] = (float)d_emis;
}

// ------------------------------------------------------------------ GVF transpose

struct GvfAdjPtrs {
    const float* lam_gl;   // [H][px]
    const float* lam_ga;   // [H][px]
    const float* lam_gn;   // [H][px]
    float* lam_lup;        // [H][px] scatter target
    float* lam_albsh;      // [H][px]
    float* lam_alb;        // [px]
    double* hour_grad;     // [H][kGFields]
};

// For every pixel p and hour: the 18 walks of the forward (first = 1,
// second = 22, the fixed 1 m case) with the coefficient of every walked
// sample in p's all-direction GVF planes; the adjoints are scattered onto the
// samples.  Samples outside the raster repeat the last in-raster sample.
template <int TY>
__global__ void __launch_bounds__(32 * TY) gvf_adjoint_kernel(SolweigScene S, const SolweigHour* __restrict__ hours,
                                                             GvfTable<22> tab, const float4* __restrict__ quads,
                                                             GvfAdjPtrs a) {
    constexpr int FIRST = 1, SECOND = 22, H = SECOND - 1;
    const int z = blockIdx.z;
    const SolweigHour& h = hours[z];
    if (!h.daytime) return;
    const long long n = (long long)S.rows * S.cols;
    const float4* quad = quads + z * n;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int pitch = 32 + 2 * H;
    float4* tile = reinterpret_cast<float4*>(smem_raw);
    const int row0 = blockIdx.y * TY - H, col0 = blockIdx.x * 32 - H;
    load_quad_tile(tile, pitch, TY + 2 * H, quad, S.rows, S.cols, row0, col0);
    __syncthreads();
    const int c = blockIdx.x * 32 + threadIdx.x;
    const int r = blockIdx.y * TY + threadIdx.y;
    if (r >= S.rows || c >= S.cols) return;
    const long long p = (long long)r * S.cols + c;
    const float4 own = tile[(threadIdx.y + H) * pitch + threadIdx.x + H];
    const bool own_ground = (__float_as_int(own.w) & kQuadGround) != 0;
    const float ob = own_ground ? 1.f : 0.f;
    const double lgl = a.lam_gl[z * n + p] / 18.0;
    const double lga = a.lam_ga[z * n + p] / 18.0;
    const double lgn = a.lam_gn[z * n + p] / 18.0;
    float* lup_t = a.lam_lup + z * n;
    float* albsh_t = a.lam_albsh + z * n;
    // own-pixel corrections (non-ground pixels)
    if (!own_ground) {
        atomicAdd(&lup_t[p], (float)(18.0 * lgl));
        atomicAdd(&albsh_t[p], (float)(18.0 * lga));
        atomicAdd(&a.lam_alb[p], (float)(18.0 * lgn));
    }
    double lwall_coef = 0.0;
    const uint32_t face = S.gvf_face[p];
    if (own_ground) {
        for (int j = 0; j < SOLWEIG_GVF_DIRECTIONS; ++j) {
            const int2* offs = tab.offs + j * SECOND;
            // pass 1: walk length, sunlit-wall statistics, frozen tail
            int hit = SECOND, n_sun = 0, n_sun_first = 0, last = -1, frozen_at = -1;
            bool seen_sun = false;
            for (int s = 0; s < SECOND; ++s) {
                const int rr = r + offs[s].x, cc = c + offs[s].y;
                const bool inside = in_raster(rr, cc, S.rows, S.cols);
                int bits;
                if (inside) {
                    bits = __float_as_int(tile[(rr - row0) * pitch + (cc - col0)].w);
                    last = s;
                } else {
                    bits = last >= 0 ? __float_as_int(tile[(r + offs[last].x - row0) * pitch + (c + offs[last].y - col0)].w) : 0;
                }
                if (!(bits & kQuadGround)) {
                    hit = s;
                    break;
                }
                seen_sun = seen_sun || (bits & kQuadSunwall);
                if (!inside) {
                    // frozen from here on: every remaining step repeats this sample
                    frozen_at = s;
                    n_sun += seen_sun ? SECOND - s : 0;
                    if (s < FIRST) n_sun_first = n_sun - (seen_sun ? SECOND - FIRST : 0);
                    break;
                }
                n_sun += seen_sun ? 1 : 0;
                if (s + 1 == FIRST) n_sun_first = n_sun;
            }
            if (hit < SECOND) {
                if (hit < FIRST) n_sun_first = n_sun + (seen_sun ? FIRST - hit : 0);
                n_sun += seen_sun ? SECOND - hit : 0;
            }
            const bool sun_near = n_sun_first > 0, sun_far = n_sun > 0;
            const int n_wall = SECOND - hit;
            const bool wall_near = FIRST > hit, wall_far = n_wall > 0;
            const bool face_drop = (n_sun == SECOND) && ((face >> j) & 1u);
            const double c1 = 0.5 / 0.9 * (sun_near ? 1.0 / (FIRST + 1) : 1.0 / FIRST);
            const double c2 = 0.4 / 0.9 * (sun_far ? 1.0 / (SECOND + 1) : 1.0 / SECOND);
            const double n1 = 0.5 / 0.9 * (wall_near ? 1.0 / (FIRST + 1) : 1.0 / FIRST);
            const double n2 = 0.4 / 0.9 * (1.0 / SECOND);
            (void)wall_far;
            // d(d_lup)/d(lwall) = c1' * n_sun_first + c2' * n_sun (when counted)
            lwall_coef += (sun_near ? 0.5 / 0.9 / (FIRST + 1) * n_sun_first : 0.0) +
                          (sun_far && !face_drop ? 0.4 / 0.9 / (SECOND + 1) * n_sun : 0.0);
            // pass 2: scatter onto the walked samples
            const int steps = frozen_at >= 0 ? frozen_at + 1 : hit;
            for (int s = 0; s < steps; ++s) {
                int rr = r + offs[s].x, cc = c + offs[s].y;
                int mult = 1;
                if (s == frozen_at) {
                    rr = r + offs[last].x;
                    cc = c + offs[last].y;
                    mult = SECOND - s;
                }
                // steps s .. s + mult - 1 all read this sample
                double k_lup = 0.0, k_nosh = 0.0;
                for (int t = s; t < s + mult; ++t) {
                    k_lup += (t < FIRST ? c1 : 0.0) + c2;
                    k_nosh += (t < FIRST ? n1 : 0.0) + n2;
                }
                const long long qq = (long long)rr * S.cols + cc;
                atomicAdd(&lup_t[qq], (float)(k_lup * lgl));
                atomicAdd(&albsh_t[qq], (float)(k_lup * lga));
                atomicAdd(&a.lam_alb[qq], (float)(k_nosh * lgn * ob));
            }
        }
    }
    if (lwall_coef != 0.0 && lgl != 0.0) {
        const double ta = h.ta, tk = ta + 273.15, tw = h.tgwall + ta + 273.15;
        const double v = lgl * lwall_coef;
        atomicAdd(&a.hour_grad[z * kGFields + kGTa], v * kSBC * 0.9 * 4.0 * (tw * tw * tw - tk * tk * tk));
        atomicAdd(&a.hour_grad[z * kGFields + kGTgwall], v * kSBC * 0.9 * 4.0 * tw * tw * tw);
    }
}

// ------------------------------------------------------------------ parameters

__global__ void param_grad_kernel(SolweigScene S, const SolweigHour* __restrict__ hours, int nhours,
                                  const float4* __restrict__ quads, const uint8_t* __restrict__ sv,
                                  const float* __restrict__ alb, const float* __restrict__ emis,
                                  const float* __restrict__ lam_lup, const float* __restrict__ lam_albsh,
                                  const float* __restrict__ lam_alb, const float* __restrict__ lam_s,
                                  const float* __restrict__ d_emis_direct, float* __restrict__ d_alb,
                                  float* __restrict__ d_emis, float* __restrict__ d_tau, double* __restrict__ hour_grad) {
    __shared__ double red[8][2];
    const long long n = (long long)S.rows * S.cols;
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const bool in = p < n;
    const long long q = in ? p : 0;
    double da = in ? lam_alb[q] : 0.0, de = in ? d_emis_direct[q] : 0.0, dt = 0.0;
    const double e = emis[q], a_ = alb[q];
    for (int hr = 0; hr < nhours; ++hr) {
        const SolweigHour& h = hours[hr];
        double g_ta = 0.0, g_ci = 0.0;
        if (h.daytime && in) {
            const long long i = hr * n + q;
            const double s = quads[i].x;
            const int vegsh = (sv[i] >> 1) & 1;
            const double ll = lam_lup[i], la = lam_albsh[i];
            const double amp = (double)S.tgk[q] * h.altmax + (double)S.tstart[q];
            const double phase =
                ((h.dectime_frac - h.snup / 24.0) / ((double)S.tmaxlst[q] / 24.0 - h.snup / 24.0)) * kPi / 2.0;
            const double wave = amp * sin(phase);
            double tg = wave * h.ci_tgg;
            const bool clamped = S.landcover == 1 && tg < 0.0;
            if (clamped) tg = 0.0;
            const double T = h.ta + 273.15, X = tg * s + T;
            const double X3 = X * X * X;
            de += ll * kSBC * (pow4(X) - pow4(T));
            da += la * s;
            dt += (ll * kSBC * e * 4.0 * X3 * tg + la * a_ + (double)lam_s[i]) * (1.0 - vegsh);
            g_ta = ll * kSBC * e * 4.0 * (X3 - T * T * T);
            g_ci = clamped ? 0.0 : ll * kSBC * e * 4.0 * X3 * s * wave;
        }
        for (int o = 16; o > 0; o >>= 1) {
            g_ta += __shfl_xor_sync(0xffffffffu, g_ta, o);
            g_ci += __shfl_xor_sync(0xffffffffu, g_ci, o);
        }
        if ((threadIdx.x & 31) == 0) {
            red[threadIdx.x >> 5][0] = g_ta;
            red[threadIdx.x >> 5][1] = g_ci;
        }
        __syncthreads();
        if (threadIdx.x < 2) {
            double v = 0.0;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) v += red[w][threadIdx.x];
            if (v != 0.0) atomicAdd(&hour_grad[hr * kGFields + (threadIdx.x == 0 ? kGTa : kGCiTgg)], v);
        }
        __syncthreads();
    }
    if (in) {
        d_alb[p] = (float)da;
        d_emis[p] = (float)de;
        d_tau[p] = (float)dt;
    }
}

// lum_grad[h][4][k]: sums over pixels of (sky, sky, veg, veg) mask bits times
// the adjoints of (luminance sum, luminance*cos*omega sum) of each mask.
__global__ void __launch_bounds__(256) lum_grad_kernel(SolweigScene S, const SolweigHour* __restrict__ hours, int nhours,
                                                       const float* __restrict__ lam_sums, double* __restrict__ lum_grad) {
    __shared__ float acc[4][kK];
    const long long n = (long long)S.rows * S.cols;
    const int z = blockIdx.y;
    if (!hours[z].daytime) return;
    for (int i = threadIdx.x; i < 4 * kK; i += blockDim.x) (&acc[0][0])[i] = 0.f;
    __syncthreads();
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
        const float l0 = lam_sums[(4LL * z) * n + p], l1 = lam_sums[(4LL * z + 1) * n + p];
        const float l2 = lam_sums[(4LL * z + 2) * n + p], l3 = lam_sums[(4LL * z + 3) * n + p];
        for (int w = 0; w < SOLWEIG_MASK_WORDS; ++w) {
            const uint32_t s = S.masks[(long long)w * n + p], v = S.masks[(long long)(SOLWEIG_MASK_WORDS + w) * n + p];
            const int nbits = S.patches - 32 * w;
            const uint32_t valid = nbits >= 32 ? 0xffffffffu : (nbits <= 0 ? 0u : ((1u << nbits) - 1u));
            for (uint32_t m = s & ~v & valid; m; m &= m - 1) {
                const int k = w * 32 + __ffs(m) - 1;
                atomicAdd(&acc[0][k], l0);
                atomicAdd(&acc[1][k], l1);
            }
            for (uint32_t m = s & v & valid; m; m &= m - 1) {
                const int k = w * 32 + __ffs(m) - 1;
                atomicAdd(&acc[2][k], l2);
                atomicAdd(&acc[3][k], l3);
            }
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < 4 * kK; i += blockDim.x) {
        const float v = (&acc[0][0])[i];
        if (v != 0.f) atomicAdd(&lum_grad[(long long)z * 4 * kK + i], (double)v);
    }
}

// ------------------------------------------------------------------ host

struct GradWork {
    long long day_total;  // the batched-day work (quads0 = its quads)
    long long quads1, sv, gvf, lam_gl, lam_ga, lam_gn, lam_s, lam_sums, lam_lup, lam_albsh, lam_alb, d_emis_direct;
    long long total;
};

GradWork grad_work_layout(long long px, int nhours) {
    GradWork g{};
    const DayWork d = day_work_layout(px, nhours, false);
    long long o = d.total;
    g.day_total = d.total;
    g.quads1 = o; o = align256(o + 16LL * px * nhours);
    g.sv = o; o = align256(o + 1LL * px * nhours);
    g.gvf = o; o = align256(o + 12LL * px * nhours);
    g.lam_gl = o; o = align256(o + 4LL * px * nhours);
    g.lam_ga = o; o = align256(o + 4LL * px * nhours);
    g.lam_gn = o; o = align256(o + 4LL * px * nhours);
    g.lam_s = o; o = align256(o + 4LL * px * nhours);
    g.lam_sums = o; o = align256(o + 16LL * px * nhours);
    g.lam_lup = o; o = align256(o + 4LL * px * nhours);
    g.lam_albsh = o; o = align256(o + 4LL * px * nhours);
    g.lam_alb = o; o = align256(o + 4LL * px);
    g.d_emis_direct = o; o = align256(o + 4LL * px);
    g.total = o;
    return g;
}

}  // namespace
}  // namespace solweig

using namespace solweig;

extern "C" int64_t solweig_day_grad_work_bytes(int rows, int cols, int nhours) {
    if (rows <= 0 || cols <= 0 || nhours <= 0) return 0;
    return grad_work_layout((long long)rows * cols, nhours).total;
}

// Shared forward of the gradient entry points: masks, parameter quads, GVF,
// contraction, tables.
static int grad_prepare(const SolweigScene* scene, const SolweigSkyLayout* layout, const SolweigHour* hours,
                        int nhours, const int32_t* gvf_dxdy, int first_steps, int second_steps,
                        const SolweigGradParams* prm, void* work, int64_t work_bytes, cudaStream_t st,
                        SolweigScene& Sp, GradWork& gw, DayWork& dw, GvfTable<22>& tab) {
    SOLWEIG_CHECK_ARG(scene && layout && hours && prm && work, "solweig_day_grad: null argument");
    SOLWEIG_CHECK_ARG(prm->albedo && prm->emissivity && prm->transmissivity, "solweig_day_grad: null parameter");
    const SolweigScene& S = *scene;
    SOLWEIG_CHECK_ARG(nhours > 0 && nhours <= kMaxGradHours, "solweig_day_grad: nhours %d outside 1..%d", nhours,
                      kMaxGradHours);
    SOLWEIG_CHECK_ARG(!S.has_water, "solweig_day_grad: scenes with water pixels are not supported");
    SOLWEIG_CHECK_ARG(S.patches == 153 || S.patches == 145, "solweig_day_grad: %d patches", S.patches);
    SOLWEIG_CHECK_ARG(first_steps == 1 && second_steps == 22 && gvf_dxdy,
                      "solweig_day_grad: only the 1 m GVF walk (first=1, second=22)");
    const long long px = (long long)S.rows * S.cols;
    gw = grad_work_layout(px, nhours);
    dw = day_work_layout(px, nhours, false);
    SOLWEIG_CHECK_ARG(work_bytes >= gw.total, "solweig_day_grad: work buffer of %lld bytes, need %lld",
                      (long long)work_bytes, gw.total);
    SOLWEIG_CHECK_ARG(((uintptr_t)work & 255) == 0, "solweig_day_grad: work buffer not 256-byte aligned");
    for (int i = 0; i < 2 * SOLWEIG_GVF_DIRECTIONS * 22; ++i)
        SOLWEIG_CHECK_ARG(gvf_dxdy[i] >= -21 && gvf_dxdy[i] <= 21, "solweig_day_grad: GVF offset outside the halo");
    char* wb = static_cast<char*>(work);
    float4* quads0 = reinterpret_cast<float4*>(wb + dw.quads);
    float4* quads1 = reinterpret_cast<float4*>(wb + gw.quads1);
    uint8_t* sv = reinterpret_cast<uint8_t*>(wb + gw.sv);
    float* gvf = reinterpret_cast<float*>(wb + gw.gvf);
    float* nosh = reinterpret_cast<float*>(wb + dw.nosh);
    float* sums = reinterpret_cast<float*>(wb + dw.sums);
    float* wf32 = reinterpret_cast<float*>(wb + dw.wf32);
    __nv_bfloat16* bw = reinterpret_cast<__nv_bfloat16*>(wb + dw.bw);
    DayTable* tables = reinterpret_cast<DayTable*>(wb + dw.tables);
    int* err = reinterpret_cast<int*>(wb + dw.error);
    cudaMemsetAsync(err, 0, sizeof(int), st);
    cudaMemsetAsync(nosh, 0, 4 * px, st);
    {
        dim3 grid(blocks_for(S.cols, 16), blocks_for(S.rows, 16), nhours);
        day_shadow_kernel<false><<<grid, dim3(16, 16), 0, st>>>(S, hours, quads0, nullptr, nullptr, nullptr,
                                                                nullptr, 0);
        SOLWEIG_CHECK_LAUNCH("day_shadow_kernel");
    }
    param_quads_kernel<<<blocks_for(px * nhours, 256), 256, 0, st>>>(S, hours, nhours, quads0, quads1, sv,
                                                                      prm->albedo, prm->emissivity,
                                                                      prm->transmissivity);
    SOLWEIG_CHECK_LAUNCH("param_quads_kernel");
    Sp = S;
    Sp.emis = prm->emissivity;
    Sp.alb = prm->albedo;
    for (int i = 0; i < SOLWEIG_GVF_DIRECTIONS * 22; ++i) {
        tab.offs[i] = make_int2(gvf_dxdy[2 * i], gvf_dxdy[2 * i + 1]);
        tab.delta[i] = gvf_dxdy[2 * i] * (32 + 42) + gvf_dxdy[2 * i + 1];
    }
    DayGvfArgs ga{1, 22, 21};
    launch_day_gvf<1, 22, 22>(16, Sp, hours, nhours, ga, tab, quads1, nullptr, gvf, nosh, st);
    SOLWEIG_CHECK_LAUNCH("day_gvf_kernel");
    const int ncols = 2 * nhours;
    const int nb = (ncols + 15) / 16 * 16;
    day_weights_kernel<<<blocks_for((long long)ncols * kK, 256), 256, 0, st>>>(layout, hours, nhours, wf32);
    split_bf16_kernel<<<blocks_for((long long)nb * kK, 256), 256, 0, st>>>(wf32, ncols, nb, S.patches, bw);
    day_tables_kernel<<<nhours, kK, 0, st>>>(layout, hours, tables);
    SOLWEIG_CHECK_LAUNCH("day_tables_kernel");
    return launch_gemm(S.masks, px, S.patches, bw, ncols, nb, sums, err, st, 0);
}

static GradPtrs grad_ptrs(void* work, const GradWork& gw, const DayWork& dw, const SolweigGradParams* prm,
                          int nhours) {
    char* wb = static_cast<char*>(work);
    GradPtrs g{};
    g.alb = prm->albedo;
    g.emis = prm->emissivity;
    g.tau = prm->transmissivity;
    g.sv = reinterpret_cast<uint8_t*>(wb + gw.sv);
    g.quads = reinterpret_cast<float4*>(wb + gw.quads1);
    g.gvf = reinterpret_cast<float*>(wb + gw.gvf);
    g.nosh = reinterpret_cast<float*>(wb + dw.nosh);
    g.sums = reinterpret_cast<float*>(wb + dw.sums);
    g.ncols = 2 * nhours;
    g.lam_gl = reinterpret_cast<float*>(wb + gw.lam_gl);
    g.lam_ga = reinterpret_cast<float*>(wb + gw.lam_ga);
    g.lam_gn = reinterpret_cast<float*>(wb + gw.lam_gn);
    g.lam_s = reinterpret_cast<float*>(wb + gw.lam_s);
    g.lam_sums = reinterpret_cast<float*>(wb + gw.lam_sums);
    g.d_emis_direct = reinterpret_cast<float*>(wb + gw.d_emis_direct);
    return g;
}

template <typename... Args>
static void launch_grad_radiation(int patches, unsigned blocks, cudaStream_t st, Args... args) {
    if (patches == 153) grad_radiation_kernel<2><<<blocks, kGradThreads, 0, st>>>(args...);
    else grad_radiation_kernel<1><<<blocks, kGradThreads, 0, st>>>(args...);
}

extern "C" int solweig_day_grad_forward(const SolweigScene* scene, const SolweigSkyLayout* layout,
                                        const SolweigHour* hours, int nhours, const int32_t* gvf_dxdy,
                                        int first_steps, int second_steps, const SolweigGradParams* params,
                                        int objective, double* daily, void* work, int64_t work_bytes, void* stream) {
    SOLWEIG_CHECK_ARG(daily && (objective == 0 || objective == 1), "solweig_day_grad_forward: bad arguments");
    cudaStream_t st = as_stream(stream);
    SolweigScene Sp;
    GradWork gw;
    DayWork dw;
    GvfTable<22> tab;
    int rc = grad_prepare(scene, layout, hours, nhours, gvf_dxdy, first_steps, second_steps, params, work,
                          work_bytes, st, Sp, gw, dw, tab);
    if (rc) return rc;
    GradPtrs g = grad_ptrs(work, gw, dw, params, nhours);
    g.daily = daily;
    g.weights = nullptr;
    g.objective = objective;
    const long long px = (long long)scene->rows * scene->cols;
    DayTable* tables = reinterpret_cast<DayTable*>(static_cast<char*>(work) + dw.tables);
    launch_grad_radiation(scene->patches, blocks_for(px, kGradThreads), st, Sp, layout, hours, nhours,
                          (const DayTable*)tables, g);
    SOLWEIG_CHECK_LAUNCH("grad_radiation_kernel");
    return SOLWEIG_OK;
}

extern "C" int solweig_day_grad_backward(const SolweigScene* scene, const SolweigSkyLayout* layout,
                                         const SolweigHour* hours, int nhours, const int32_t* gvf_dxdy,
                                         int first_steps, int second_steps, const SolweigGradParams* params,
                                         int objective, const float* weights, float* d_albedo,
                                         float* d_emissivity, float* d_transmissivity, double* hour_grad,
                                         double* lum_grad, void* work, int64_t work_bytes, void* stream) {
    SOLWEIG_CHECK_ARG(weights && d_albedo && d_emissivity && d_transmissivity && hour_grad && lum_grad &&
                          (objective == 0 || objective == 1),
                      "solweig_day_grad_backward: bad arguments");
    cudaStream_t st = as_stream(stream);
    SolweigScene Sp;
    GradWork gw;
    DayWork dw;
    GvfTable<22> tab;
    int rc = grad_prepare(scene, layout, hours, nhours, gvf_dxdy, first_steps, second_steps, params, work,
                          work_bytes, st, Sp, gw, dw, tab);
    if (rc) return rc;
    const long long px = (long long)scene->rows * scene->cols;
    char* wb = static_cast<char*>(work);
    GradPtrs g = grad_ptrs(work, gw, dw, params, nhours);
    g.daily = nullptr;
    g.weights = weights;
    g.objective = objective;
    g.hour_grad = hour_grad;
    cudaMemsetAsync(hour_grad, 0, sizeof(double) * kGFields * nhours, st);
    cudaMemsetAsync(lum_grad, 0, sizeof(double) * 4 * kK * nhours, st);
    cudaMemsetAsync(wb + gw.lam_lup, 0, 4LL * px * nhours, st);
    cudaMemsetAsync(wb + gw.lam_albsh, 0, 4LL * px * nhours, st);
    cudaMemsetAsync(wb + gw.lam_alb, 0, 4LL * px, st);
    DayTable* tables = reinterpret_cast<DayTable*>(wb + dw.tables);
    launch_grad_radiation(scene->patches, blocks_for(px, kGradThreads), st, Sp, layout, hours, nhours,
                          (const DayTable*)tables, g);
    SOLWEIG_CHECK_LAUNCH("grad_radiation_kernel");
    GvfAdjPtrs ap{g.lam_gl, g.lam_ga, g.lam_gn, reinterpret_cast<float*>(wb + gw.lam_lup),
                  reinterpret_cast<float*>(wb + gw.lam_albsh), reinterpret_cast<float*>(wb + gw.lam_alb), hour_grad};
    {
        constexpr int TY = 8;
        const size_t smem = sizeof(float4) * (size_t)(32 + 42) * (TY + 42);
        set_smem_attr((const void*)gvf_adjoint_kernel<TY>, smem);
        dim3 grid(blocks_for(scene->cols, 32), blocks_for(scene->rows, TY), nhours);
        gvf_adjoint_kernel<TY><<<grid, dim3(32, TY), smem, st>>>(Sp, hours, tab, g.quads, ap);
        SOLWEIG_CHECK_LAUNCH("gvf_adjoint_kernel");
    }
    param_grad_kernel<<<blocks_for(px, 256), 256, 0, st>>>(
        Sp, hours, nhours, g.quads, g.sv, params->albedo, params->emissivity, ap.lam_lup, ap.lam_albsh,
        ap.lam_alb, g.lam_s, g.d_emis_direct, d_albedo, d_emissivity, d_transmissivity, hour_grad);
    SOLWEIG_CHECK_LAUNCH("param_grad_kernel");
    {
        dim3 grid(148, nhours);
        lum_grad_kernel<<<grid, 256, 0, st>>>(Sp, hours, nhours, g.lam_sums, lum_grad);
        SOLWEIG_CHECK_LAUNCH("lum_grad_kernel");
    }
    return SOLWEIG_OK;
}
