// The hourly SOLWEIG step: two kernels per daytime hour, one per night hour.
//
//  K1 step_shadow_kernel   shadow sweep + per-pixel GVF inputs -> float4 quad
//                          (shadow, Lup, albedo, ground|sunwall bits)
//  K2 step_radiation_kernel<Day>
//                          GVF over a shared-memory quad tile, wave delay of
//                          the thermal state, F_sh, K/L fluxes with the
//                          anisotropic patch sums, Tmrt and UTCI
//
// Per-pixel arithmetic outside the GVF walk and the patch loop is float64
// (B200 runs FP64 at half the FP32 rate, and it is a few hundred operations
// per pixel-hour); stored planes are float32.
#include "gvf_fields.cuh"
#include "hour.cuh"
#include "radiation.cuh"

namespace solweig {

constexpr int kStepBX = 32, kStepBY = 8;

__global__ void __launch_bounds__(kStepBX* kStepBY) step_shadow_kernel(
    SolweigScene S, const SolweigHour* __restrict__ hours, int hour, float4* __restrict__ quad,
    float* __restrict__ lup_first) {
    const SolweigHour& h = hours[hour];
    if (!h.daytime) return;
    const int c = blockIdx.x * kStepBX + threadIdx.x;
    const int r = blockIdx.y * kStepBY + threadIdx.y;
    if (r >= S.rows || c >= S.cols) return;
    shadow_quad_pixel(S, h, r, c, quad, lup_first);
}

struct StepGvfArgs {
    const int2* offs;  // [18][second]
    int first, second, halo;
};

// Ground view factors of one daytime hour: the 15 planes [15][pixels]
// (Lup, albedo, albedo without shadow) x (all, E, S, W, N), ambient and own-pixel
// corrections included.  FIXED > 0: walk length and `first` fixed at compile
// time (FIRST, SECOND); otherwise the runtime values of `ga` are used.
template <int TY, int FIRST, int SECOND, int TABLE, bool WATER>
__global__ void __launch_bounds__(32 * TY) step_gvf_kernel(
    SolweigScene S, const SolweigHour* __restrict__ hours, int hour, StepGvfArgs ga,
    GvfTable<TABLE> tab, const float4* __restrict__ quad, const float* __restrict__ lup_first,
    float* __restrict__ gvf) {
    const SolweigHour& h = hours[hour];
    if (!h.daytime) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int H = ga.halo, second = ga.second, first = ga.first;
    const int pitch = 32 + 2 * H;
    float4* tile = reinterpret_cast<float4*>(smem_raw);
    const int row0 = blockIdx.y * TY - H, col0 = blockIdx.x * 32 - H;
    load_quad_tile(tile, pitch, TY + 2 * H, quad, S.rows, S.cols, row0, col0);
    __syncthreads();
    const int c = blockIdx.x * 32 + threadIdx.x;
    const int r = blockIdx.y * TY + threadIdx.y;
    if (r >= S.rows || c >= S.cols) return;
    const long long n = (long long)S.rows * S.cols;
    const long long p = (long long)r * S.cols + c;
    const float4* own_cell = tile + (threadIdx.y + H) * pitch + threadIdx.x + H;
    const float4 own = *own_cell;
    const double ta = h.ta;
    const float lwall = (float)(kSBC * 0.9 * pow4(h.tgwall + ta + 273.15) - kSBC * 0.9 * pow4(ta + 273.15));
    const float albedo_b = 0.2f;
    const uint32_t face = S.gvf_face[p];
    float lup[5], alb[5], nosh[5];
    const bool own_ground = (__float_as_int(own.w) & kQuadGround) != 0;
    if (WATER) {
        // Rare path (water pixels change the first direction's Lup): general walk.
        GvfScalars gs{lwall, albedo_b, first, second};
        auto sample = [&](int rr, int cc) -> float4 { return tile[(rr - row0) * pitch + (cc - col0)]; };
        auto lfirst = [&](int rr, int cc) -> float { return __ldg(&lup_first[(long long)rr * S.cols + cc]); };
        const GvfSums g = gvf_walk(sample, lfirst, true, r, c, S.rows, S.cols, tab.offs, face, own, gs);
        for (int d = 0; d < 5; ++d) {
            lup[d] = g.lup[d];
            alb[d] = g.alb[d];
            nosh[d] = g.nosh[d];
        }
    } else {
#pragma unroll
        for (int d = 0; d < 5; ++d) lup[d] = alb[d] = nosh[d] = 0.f;
        const bool interior = row0 >= 0 && col0 >= 0 && row0 + TY + 2 * H <= S.rows &&
                              col0 + pitch <= S.cols;
        const float inv_first = 1.f / first, inv_first1 = 1.f / (first + 1);
        const float inv_second = 1.f / second, inv_second1 = 1.f / (second + 1);
#pragma unroll 1
        for (int j = 0; j < SOLWEIG_GVF_DIRECTIONS; ++j) {
            const bool fj = (face >> j) & 1u;
            const int base = j * (SECOND > 0 ? SECOND : second);
            GvfDir d;
            if (SECOND > 0) {
                d = interior ? gvf_direction_fixed<true, FIRST, SECOND>(own_cell, tab.delta + base, tab.offs + base, r, c,
                                                                        S.rows, S.cols, own_ground, lwall, albedo_b, fj)
                             : gvf_direction_fixed<false, FIRST, SECOND>(own_cell, tab.delta + base, tab.offs + base, r, c,
                                                                         S.rows, S.cols, own_ground, lwall, albedo_b, fj);
            } else {
                d = interior ? gvf_direction<true>(own_cell, tab.delta + base, tab.offs + base, r, c, S.rows,
                                                   S.cols, own_ground, first, second, inv_first, inv_first1,
                                                   inv_second, inv_second1, lwall, albedo_b, fj)
                             : gvf_direction<false>(own_cell, tab.delta + base, tab.offs + base, r, c, S.rows,
                                                    S.cols, own_ground, first, second, inv_first, inv_first1,
                                                    inv_second, inv_second1, lwall, albedo_b, fj);
            }
            const unsigned groups = gvf_direction_groups(j);
#pragma unroll
            for (int k = 0; k < 5; ++k)
                if (groups & (1u << k)) {
                    lup[k] += d.lup;
                    alb[k] += d.alb;
                    nosh[k] += d.nosh;
                }
        }
        // own-pixel corrections (added once per direction in the reference)
        const float ob = own_ground ? 1.f : 0.f;
#pragma unroll
        for (int k = 0; k < 5; ++k) {
            const float cnt = k == 0 ? 18.f : 9.f;
            nosh[k] *= ob;
            lup[k] += cnt * (own.y * (1.f - ob));
            alb[k] += cnt * (own.z * (1.f - ob) * own.x);
            nosh[k] += cnt * (own.z * (1.f - ob));
        }
    }
    const double ambient = kSBC * (double)S.emis[p] * pow4(ta + 273.15);
#pragma unroll
    for (int k = 0; k < 5; ++k) {
        const float div = k == 0 ? 18.f : 9.f;
        gvf[(long long)k * n + p] = (float)((double)(lup[k] / div) + ambient);
        gvf[(long long)(5 + k) * n + p] = alb[k] / div;
        gvf[(long long)(10 + k) * n + p] = nosh[k] / div;
    }
}

size_t gvf_smem_bytes(int halo, int ty) {
    return sizeof(float4) * (size_t)(32 + 2 * halo) * (ty + 2 * halo);
}

__device__ __forceinline__ float* state_plane(const SolweigState& st, int d) {
    return d == 0 ? st.tgmap1 : d == 1 ? st.tgmap1e : d == 2 ? st.tgmap1s : d == 3 ? st.tgmap1w : st.tgmap1n;
}

__device__ __forceinline__ float* kside_plane(const SolweigOutputs& o, int d) {
    return d == 1 ? o.keast : d == 2 ? o.ksouth : d == 3 ? o.kwest : o.knorth;
}

__device__ __forceinline__ float* lcard_plane(const SolweigOutputs& o, int d) {
    return d == 1 ? o.least : d == 2 ? o.lsouth : d == 3 ? o.lwest : o.lnorth;
}

// Radiation epilogue of one pixel-hour.  The 15 GVF planes are consumed one
// direction at a time (Kup and the delayed Lup of that direction) so only the
// sums Tmrt needs stay live: all-direction values and the sum over E, S, W, N.
template <bool Day, bool Cardinal>
__device__ __forceinline__ void radiation_body(
    const SolweigScene& S, const SolweigSkyLayout& L, const SolweigHour& h, const SolweigState& st,
    const SolweigOutputs& out, const float4* __restrict__ quad, const float* __restrict__ gvfp) {
    __shared__ PatchSmem ps;
    stage_patches(ps, L, h);
    __syncthreads();
    const int c = blockIdx.x * kStepBX + threadIdx.x;
    const int r = blockIdx.y * kStepBY + threadIdx.y;
    if (r >= S.rows || c >= S.cols) return;
    const long long n = (long long)S.rows * S.cols;
    const long long p = (long long)r * S.cols + c;
    const uint8_t fl = S.flags[p];
    const bool ground = fl & 1;
    const double ta = h.ta;
    const double tk = ta + 273.15;
    const double emis = S.emis[p];
    constexpr double ewall = 0.9, albedo_b = 0.2;
    constexpr double absK = 0.7, absL = 0.95, Fside = 0.22, Fup = 0.06, Fcyl = 0.28;

    // --- anisotropic patch sums (sky / vegetation luminance, building split)
    uint32_t Sw[SOLWEIG_MASK_WORDS], Vw[SOLWEIG_MASK_WORDS];
#pragma unroll
    for (int w = 0; w < SOLWEIG_MASK_WORDS; ++w) {
        Sw[w] = S.masks[(long long)w * n + p];
        Vw[w] = S.masks[(long long)(SOLWEIG_MASK_WORDS + w) * n + p];
    }
    const PatchSums pz = patch_loop<Cardinal>(ps, Sw, Vw, S.tan_asvf[p], Day);
    double ld_sky = 0.0, ls_sky = 0.0;
    for (int b = 0; b < L.nbands; ++b) {
        const double cnt = S.sky_band_counts[(long long)b * n + p];
        ld_sky += (double)ps.band_down[b] * cnt;
        ls_sky += (double)ps.band_side[b] * cnt;
    }
    const double lw_shade = (ewall * kSBC * pow4(tk)) / kPi;
    const double lw_sun = Day ? (ewall * kSBC * pow4(ta + h.tgwall + 273.15)) / kPi : 0.0;

    double shadow = 0.0, tg = 0.0, tg_out = ta;
    double kup_all = 0.0, kup_card = 0.0, lup_all, lup_card = 0.0;
    double kdown = 0.0, kside = 0.0, kside_i = 0.0, kside_d = 0.0, d_rad = 0.0;
    double refl;
    if (Day) {
        shadow = quad[p].x;
        const double fsh = wedge_fsh(S.svfalfa[p], h.tan_zen);
        const double svfbuveg = S.svfbuveg[p];
        const double reflected = albedo_b * (1.0 - svfbuveg) * (h.rad_g * (1.0 - fsh) + h.rad_d * fsh);
        const double base_up = h.rad_d * svfbuveg + reflected;
        const double direct_up = h.rad_i * h.sin_alt;
#pragma unroll
        for (int d = 0; d < 5; ++d) {
            const double g_lup = gvfp[(long long)d * n + p];
            const double g_alb = gvfp[(long long)(5 + d) * n + p];
            const double g_nosh = gvfp[(long long)(10 + d) * n + p];
            const double kup = g_alb * direct_up + base_up * g_nosh;
            float* sp = state_plane(st, d);
            const double prev = h.firstdaytime ? g_lup : (double)sp[p];
            const double lup = g_lup * (1.0 - h.wave_weight) + prev * h.wave_weight;
            sp[p] = (float)(h.wave_update ? lup : prev);
            if (d == 0) {
                kup_all = kup;
                lup_all = lup;
                if (out.kup) out.kup[p] = (float)kup;
                if (out.lup) out.lup[p] = (float)lup;
            } else {
                kup_card += kup;
                lup_card += lup;
                float* ko = kside_plane(out, d);
                if (ko) ko[p] = (float)(kup * 0.5);
                float* lo = lcard_plane(out, d);
                if (lo) lo[p] = (float)(lup * 0.5);  // cardinal patch terms added below
            }
        }
        tg = ground_tg(S, h, p);
        if (S.has_water && (fl & 4)) tg = h.twater - ta;
        {
            const double cur = tg * shadow + ta;
            const double prev = h.firstdaytime ? cur : (double)st.tgout1[p];
            tg_out = cur * (1.0 - h.wave_weight) + prev * h.wave_weight;
            st.tgout1[p] = (float)(h.wave_update ? tg_out : prev);
        }
        const double dsh_veg = 1.0 - (1.0 - 0.03);
        d_rad = h.rad_d * ((double)pz.lum_sky + dsh_veg * (double)pz.lum_veg);
        kdown = h.rad_i * shadow * h.sin_alt + d_rad + reflected;
        kside_i = shadow * h.rad_i * h.cos_alt;
        kside_d = (h.rad_d / h.rad_tot) * ((double)pz.cw_sky + dsh_veg * (double)pz.cw_veg);
        const double sw_shade = (albedo_b * h.rad_d * 0.5) / kPi;
        const double sw_sun = (albedo_b * (h.rad_i * h.cos_alt) + h.rad_d * 0.5) / kPi;
        kside = kside_i + kside_d + sw_sun * (double)pz.sw_sun + sw_shade * (double)pz.sw_shade +
                sw_shade * (double)S.veg_sums[p];
    } else {
        double lup = kSBC * emis * pow4(ta + 0.0 + 273.15);
        if (S.landcover == 1 && (fl & 4)) lup = kSBC * 0.98 * pow4(h.twater + 273.15);
        lup_all = lup;
        lup_card = 4.0 * lup;
        if (out.lup) out.lup[p] = (float)lup;
        for (int d = 1; d < 5; ++d) {
            float* ko = kside_plane(out, d);
            if (ko) ko[p] = 0.f;
            float* lo = lcard_plane(out, d);
            if (lo) lo[p] = (float)(lup * 0.5);
        }
        if (out.kup) out.kup[p] = 0.f;
    }
    refl = ((ld_sky + lup_all) * (1.0 - ewall) * 0.5) / kPi;
    const double vc = S.veg_sums[p], vs = S.veg_sums[n + p];
    const double oc = S.veg_sums[2 * n + p], os = S.veg_sums[3 * n + p];
    const double ldown = ld_sky + lw_shade * vs + lw_shade * (double)pz.lw_shade_s +
                         lw_sun * (double)pz.lw_sun_s + refl * os;
    const double lside = ls_sky + lw_shade * vc + lw_shade * (double)pz.lw_shade_c +
                         lw_sun * (double)pz.lw_sun_c + refl * oc;
    if (Cardinal) {
#pragma unroll
        for (int d = 1; d < 5; ++d) {
            float* lo = lcard_plane(out, d);
            if (lo)
                lo[p] += (float)((double)pz.card_sky[d - 1] + lw_shade * (double)pz.card_veg[d - 1] +
                                 lw_sun * (double)pz.card_sun[d - 1] +
                                 lw_shade * (double)pz.card_shade[d - 1] +
                                 refl * (double)pz.card_obst[d - 1]);
        }
    }
    // Tmrt (cylinder, anisotropic sky): Keast.. = KupE..*0.5, Least.. = LupE..*0.5
    const double sstr = absK * (kside * Fcyl + (kdown + kup_all) * Fup + 0.5 * kup_card * Fside) +
                        absL * ((ldown + lup_all) * Fup + lside * Fcyl + 0.5 * lup_card * Fside);
    const double tmrt = sqrt(sqrt(sstr / (absL * kSBC))) - 273.2;
    if (out.tmrt) out.tmrt[p] = (float)tmrt;
    if (out.utci) out.utci[p] = ground ? utci_eval(h.utci, tmrt, ta, h.utci_valid) : __int_as_float(0x7fc00000);
    if (out.ldown) out.ldown[p] = (float)ldown;
    if (out.lside) out.lside[p] = (float)lside;
    if (out.kdown) out.kdown[p] = (float)kdown;
    if (out.kside_i) out.kside_i[p] = (float)kside_i;
    if (out.kside_d) out.kside_d[p] = (float)kside_d;
    if (out.kside) out.kside[p] = (float)kside;
    if (out.d_rad) out.d_rad[p] = (float)d_rad;
    if (out.shadow) out.shadow[p] = (float)shadow;
    if (out.tg) out.tg[p] = (float)tg;
    if (out.tg_out) out.tg_out[p] = (float)tg_out;
}

// One kernel for both branches: the day/night choice is read from the hour
// record in device memory, so a captured day replays for any forcing.
template <bool Cardinal>
__global__ void __launch_bounds__(kStepBX* kStepBY, 3) step_radiation_kernel(
    SolweigScene S, const SolweigSkyLayout* __restrict__ L, const SolweigHour* __restrict__ hours,
    int hour, SolweigState st, SolweigOutputs out, const float4* __restrict__ quad,
    const float* __restrict__ gvfp) {
    const SolweigHour& h = hours[hour];
    if (h.daytime)
        radiation_body<true, Cardinal>(S, *L, h, st, out, quad, gvfp);
    else
        radiation_body<false, Cardinal>(S, *L, h, st, out, quad, gvfp);
}


}  // namespace solweig

using namespace solweig;

static int check_scene(const SolweigScene* S) {
    SOLWEIG_CHECK_ARG(S, "null scene");
    SOLWEIG_CHECK_ARG(S->rows > 0 && S->cols > 0 && S->rows < (1 << 20) && S->cols < (1 << 20),
                      "bad scene shape %dx%d", S->rows, S->cols);
    SOLWEIG_CHECK_ARG(S->dsm && S->vegdem && S->vegdem2 && S->walls && S->aspect && S->flags &&
                          S->alb && S->emis && S->tgk && S->tstart && S->tmaxlst && S->svfbuveg &&
                          S->svfalfa && S->tan_asvf && S->masks && S->veg_sums &&
                          S->sky_band_counts && S->gvf_face,
                      "scene has a null array");
    return SOLWEIG_OK;
}

static void set_smem_once(const void* kernel, size_t bytes) {
    // cudaFuncSetAttribute is not a stream operation; remember the largest
    // size set per kernel so steady-state launches (and graph capture) skip it.
    static thread_local const void* which[32] = {};
    static thread_local size_t done[32] = {};
    int slot = -1;
    for (int i = 0; i < 32; ++i) {
        if (which[i] == kernel) {
            if (done[i] >= bytes) return;
            slot = i;
            break;
        }
        if (!which[i] && slot < 0) slot = i;
    }
    cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (slot >= 0) {
        which[slot] = kernel;
        done[slot] = bytes;
    }
}

extern "C" int solweig_step_shadow(const SolweigScene* scene, const SolweigHour* hours, int hour,
                                   float* scratch, void* stream) {
    int rc = check_scene(scene);
    if (rc) return rc;
    SOLWEIG_CHECK_ARG(hours && hour >= 0 && scratch, "solweig_step_shadow: bad arguments");
    const SolweigScene& S = *scene;
    dim3 block(kStepBX, kStepBY);
    dim3 grid(blocks_for(S.cols, kStepBX), blocks_for(S.rows, kStepBY));
    float4* quad = reinterpret_cast<float4*>(scratch);
    float* lup_first = S.has_water ? scratch + 4 * (long long)S.rows * S.cols : nullptr;
    step_shadow_kernel<<<grid, block, 0, as_stream(stream)>>>(S, hours, hour, quad, lup_first);
    SOLWEIG_CHECK_LAUNCH("step_shadow_kernel");
    return SOLWEIG_OK;
}

// scratch layout [20][pixels]: quad (4 planes as float4), lup_first (1), gvf (15)
static inline float4* scratch_quad(float* scratch) { return reinterpret_cast<float4*>(scratch); }
static inline float* scratch_lup_first(float* scratch, long long n) { return scratch + 4 * n; }
static inline float* scratch_gvf(float* scratch, long long n) { return scratch + 5 * n; }

template <int TY, int FIRST, int SECOND, int TABLE>
static void launch_gvf(const SolweigScene& S, const SolweigHour* hours, int hour, const StepGvfArgs& ga,
                       const GvfTable<TABLE>& tab, float* scratch, size_t smem, cudaStream_t st) {
    const long long n = (long long)S.rows * S.cols;
    const float* lup_first = S.has_water ? scratch_lup_first(scratch, n) : nullptr;
    dim3 grid(blocks_for(S.cols, 32), blocks_for(S.rows, TY));
    if (S.has_water) {
        auto k = step_gvf_kernel<TY, FIRST, SECOND, TABLE, true>;
        set_smem_once((const void*)k, smem);
        k<<<grid, dim3(32, TY), smem, st>>>(S, hours, hour, ga, tab, scratch_quad(scratch), lup_first,
                                            scratch_gvf(scratch, n));
    } else {
        auto k = step_gvf_kernel<TY, FIRST, SECOND, TABLE, false>;
        set_smem_once((const void*)k, smem);
        k<<<grid, dim3(32, TY), smem, st>>>(S, hours, hour, ga, tab, scratch_quad(scratch), lup_first,
                                            scratch_gvf(scratch, n));
    }
}

template <int TABLE>
static void fill_table(GvfTable<TABLE>& tab, const int32_t* dxdy, int second, int pitch) {
    for (int i = 0; i < SOLWEIG_GVF_DIRECTIONS * second; ++i) {
        tab.offs[i] = make_int2(dxdy[2 * i], dxdy[2 * i + 1]);
        tab.delta[i] = dxdy[2 * i] * pitch + dxdy[2 * i + 1];
    }
}

extern "C" int solweig_step_gvf(const SolweigScene* scene, const SolweigHour* hours, int hour,
                                const int32_t* gvf_dxdy_host, int first_steps, int second_steps,
                                float* scratch, int tile_rows, void* stream) {
    int rc = check_scene(scene);
    if (rc) return rc;
    SOLWEIG_CHECK_ARG(hours && hour >= 0 && scratch && gvf_dxdy_host, "solweig_step_gvf: bad arguments");
    SOLWEIG_CHECK_ARG(second_steps >= 1 && second_steps <= SOLWEIG_GVF_MAX_STEPS && first_steps >= 1 &&
                          first_steps <= second_steps,
                      "solweig_step_gvf: GVF steps first=%d second=%d", first_steps, second_steps);
    SOLWEIG_CHECK_ARG(tile_rows == 4 || tile_rows == 8 || tile_rows == 16,
                      "solweig_step_gvf: tile_rows must be 4, 8 or 16");
    const SolweigScene& S = *scene;
    StepGvfArgs ga{nullptr, first_steps, second_steps, second_steps - 1};
    const int pitch = 32 + 2 * ga.halo;
    for (int i = 0; i < 2 * SOLWEIG_GVF_DIRECTIONS * second_steps; ++i)
        SOLWEIG_CHECK_ARG(gvf_dxdy_host[i] >= -ga.halo && gvf_dxdy_host[i] <= ga.halo,
                          "solweig_step_gvf: offset %d outside the halo %d", gvf_dxdy_host[i], ga.halo);
    const size_t smem = gvf_smem_bytes(ga.halo, tile_rows);
    SOLWEIG_CHECK_ARG(smem <= 227 * 1024, "solweig_step_gvf: GVF halo %d too large", ga.halo);
    cudaStream_t st = as_stream(stream);
    if (first_steps == 1 && second_steps == 22) {
        GvfTable<22> tab;
        fill_table(tab, gvf_dxdy_host, 22, pitch);
        if (tile_rows == 4) launch_gvf<4, 1, 22, 22>(S, hours, hour, ga, tab, scratch, smem, st);
        else if (tile_rows == 8) launch_gvf<8, 1, 22, 22>(S, hours, hour, ga, tab, scratch, smem, st);
        else launch_gvf<16, 1, 22, 22>(S, hours, hour, ga, tab, scratch, smem, st);
    } else {
        GvfTable<SOLWEIG_GVF_MAX_STEPS> tab;
        fill_table(tab, gvf_dxdy_host, second_steps, pitch);
        if (tile_rows == 4) launch_gvf<4, 0, 0, SOLWEIG_GVF_MAX_STEPS>(S, hours, hour, ga, tab, scratch, smem, st);
        else if (tile_rows == 8) launch_gvf<8, 0, 0, SOLWEIG_GVF_MAX_STEPS>(S, hours, hour, ga, tab, scratch, smem, st);
        else launch_gvf<16, 0, 0, SOLWEIG_GVF_MAX_STEPS>(S, hours, hour, ga, tab, scratch, smem, st);
    }
    SOLWEIG_CHECK_LAUNCH("step_gvf_kernel");
    return SOLWEIG_OK;
}

extern "C" int solweig_step_radiation(const SolweigScene* scene, const SolweigSkyLayout* layout,
                                      const SolweigHour* hours, int hour, const SolweigState* state,
                                      const SolweigOutputs* out, float* scratch, void* stream) {
    int rc = check_scene(scene);
    if (rc) return rc;
    SOLWEIG_CHECK_ARG(layout && hours && hour >= 0 && state && out && scratch,
                      "solweig_step_radiation: null argument");
    SOLWEIG_CHECK_ARG(state->tgmap1 && state->tgmap1e && state->tgmap1s && state->tgmap1w &&
                          state->tgmap1n && state->tgout1,
                      "solweig_step_radiation: state has a null plane");
    const SolweigScene& S = *scene;
    const long long n = (long long)S.rows * S.cols;
    const bool full = out->least || out->lsouth || out->lwest || out->lnorth;
    dim3 block(kStepBX, kStepBY);
    dim3 grid(blocks_for(S.cols, kStepBX), blocks_for(S.rows, kStepBY));
    cudaStream_t st = as_stream(stream);
    if (full)
        step_radiation_kernel<true><<<grid, block, 0, st>>>(S, layout, hours, hour, *state, *out,
                                                           scratch_quad(scratch), scratch_gvf(scratch, n));
    else
        step_radiation_kernel<false><<<grid, block, 0, st>>>(S, layout, hours, hour, *state, *out,
                                                            scratch_quad(scratch), scratch_gvf(scratch, n));
    SOLWEIG_CHECK_LAUNCH("step_radiation_kernel");
    return SOLWEIG_OK;
}

extern "C" int solweig_step(const SolweigScene* scene, const SolweigSkyLayout* layout,
                            const SolweigHour* hours, int hour, const SolweigState* state,
                            const SolweigOutputs* out, const int32_t* gvf_dxdy, int first_steps,
                            int second_steps, float* scratch, void* stream) {
    int rc = solweig_step_shadow(scene, hours, hour, scratch, stream);
    if (rc) return rc;
    rc = solweig_step_gvf(scene, hours, hour, gvf_dxdy, first_steps, second_steps, scratch, 8, stream);
    if (rc) return rc;
    return solweig_step_radiation(scene, layout, hours, hour, state, out, scratch, stream);
}

extern "C" int solweig_day(const SolweigScene* scene, const SolweigSkyLayout* layout,
                           const SolweigHour* hours, int nhours, const SolweigState* state,
                           const SolweigOutputs* base, int64_t hour_stride,
                           const int32_t* gvf_dxdy, int first_steps, int second_steps,
                           float* scratch, void* stream) {
    SOLWEIG_CHECK_ARG(base && nhours > 0 && hour_stride >= 0, "solweig_day: bad arguments");
    for (int hr = 0; hr < nhours; ++hr) {
        SolweigOutputs o = *base;
        float** f = reinterpret_cast<float**>(&o);
        const int nf = sizeof(SolweigOutputs) / sizeof(float*);
        for (int i = 0; i < nf; ++i)
            if (f[i]) f[i] += (long long)hr * hour_stride;
        int rc = solweig_step(scene, layout, hours, hr, state, &o, gvf_dxdy, first_steps,
                              second_steps, scratch, stream);
        if (rc) return rc;
    }
    return SOLWEIG_OK;
}
