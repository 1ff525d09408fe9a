// The batched form of a SOLWEIG day: all hours of one day in a few launches
// (instead of three per hour), with the luminance-weighted patch sums of all
// hours as one BF16 tensor-core contraction.  The sweep stage can be issued
// in hour ranges (solweig_day_batched_part) while the host plans later hours.
//
//  0 ceiling_dilate_kernel  once per day: height planes dilated along rows /
//                           columns; day_ray_ceiling_kernel, grid.z = hour:
//                           upper bounds of the heights ahead along the sun
//                           ray (early exit of the sweep);
//                           day_ray_exits_kernel: first step outside the
//                           raster of every row and column
//  1 day_shadow_kernel      grid.z = hour: shadow sweep + GVF field quads
//                           (day_sweep_tma_kernel with sweep_window = 1 / 2:
//                           the same sweep on TMA-staged shared-memory windows
//                           with the warp-vote exit, sweep_tma.cuh)
//  2 day_gvf_hv_kernel      32 x 32 tiles, every daytime hour per block (4 per
//                           shared-memory pass): all-direction GVF (Lup,
//                           albedo) + the pixel's shadow, the hour-independent
//                           albedo-without-shadow GVF once per day
//                           (day_gvf_kernel, grid.z = hour, for other walk
//                           lengths and water scenes)
//  3 day_weights_kernel     per-hour patch weights (luminance, luminance*cos*omega)
//  4 split_bf16_kernel      weights (and 0.03 x the weights) -> BF16 hi/lo
//                           pairs in the canonical K-major shared-memory
//                           layout of the contraction
//  5 day_tables_kernel      per hour: exact thresholds on tan(asvf) for the
//                           sunlit / shaded split of building patches, sorted,
//                           with the prefix/suffix patch masks, bucket start
//                           tables and the hour's flux scalars
//  6 patch_gemm_kernel      tcgen05: [128 px x 160 patches] 0/1 sky masks x
//                           [160 x 2H] weights + vegetation masks x 0.03 x
//                           weights into one set of FP32 columns in tensor memory
//  7 day_radiation_kernel   one thread per pixel loops over the hours: wave
//                           delay state in registers, fluxes, Tmrt, UTCI
//
// Two identities of the reference model make the hour loop cheap:
//  * each GVF search direction belongs to exactly two of the E/S/W/N groups
//    and the group means divide by 9 (all directions: by 18), so
//    sum(E,S,W,N) of every GVF plane -- and of Kup, Lup and their delayed
//    state -- is exactly 4x the all-direction value; Tmrt only needs that sum
//    (src/umep_solweig.py:345-360), so only the all-direction planes are made;
//  * the GVF albedo-without-shadow plane depends on the walk geometry and
//    the albedo only, so it is computed once per day.
// The building-patch split of Kside_veg_v2022a / Lcyl_v2022a
// (src/umep_solweig.py:1362-1397) compares fl(tan(asvf) + yi_k) against
// fixed per-patch limits; for each patch and hour that is equivalent to one
// compare of tan(asvf) with a float64 threshold found by bisection over the
// doubles, so a pixel-hour needs two short scans from a 256-bucket start
// table and band popcounts instead of a loop over its building patches.
#include "day_kernels.cuh"

using namespace solweig;

extern "C" int64_t solweig_day_batched_work_bytes(int rows, int cols, int nhours, int has_water) {
    if (rows <= 0 || cols <= 0 || nhours <= 0) return 0;
    return day_work_layout((long long)rows * cols, nhours, has_water != 0).total;
}

extern "C" int solweig_day_batched_layout(int rows, int cols, int nhours, int has_water, int64_t* offsets) {
    SOLWEIG_CHECK_ARG(offsets && rows > 0 && cols > 0 && nhours > 0, "solweig_day_batched_layout: bad arguments");
    const DayWork w = day_work_layout((long long)rows * cols, nhours, has_water != 0);
    const long long v[11] = {w.quads, w.lup_first, w.gvf, w.nosh, w.sums, w.wf32, w.bw, w.tables, w.error,
                             w.tilemax, w.total};
    for (int i = 0; i < 11; ++i) offsets[i] = v[i];
    return SOLWEIG_OK;
}

extern "C" int solweig_gvf_statics(const SolweigScene* scene, const int32_t* gvf_dxdy, int first_steps,
                                   int second_steps, uint32_t* hits, float* nosh, void* stream) {
    SOLWEIG_CHECK_ARG(scene && gvf_dxdy && hits && nosh, "solweig_gvf_statics: null argument");
    SOLWEIG_CHECK_ARG(first_steps == 1 && second_steps == 22,
                      "solweig_gvf_statics: only the 1 m walk (first 1, second 22), not %d/%d", first_steps,
                      second_steps);
    SOLWEIG_CHECK_ARG(!scene->has_water, "solweig_gvf_statics: scenes with water walk per hour");
    SOLWEIG_CHECK_ARG(scene->rows > 0 && scene->cols > 0 && scene->flags && scene->alb,
                      "solweig_gvf_statics: bad scene");
    const SolweigScene& S = *scene;
    GvfTable<22> tab;
    fill_day_table(tab, gvf_dxdy, 22, kHvPitch);
    cudaStream_t st = as_stream(stream);
    const size_t smem = gvf_statics_smem_bytes();
    set_smem_attr((const void*)gvf_statics_kernel, smem);
    dim3 grid(blocks_for(S.cols, kHvTile), blocks_for(S.rows, kHvTile));
    gvf_statics_kernel<<<grid, dim3(kHvTile, kHvTile), smem, st>>>(S, tab, hits, nosh);
    SOLWEIG_CHECK_LAUNCH("gvf_statics_kernel");
    return SOLWEIG_OK;
}

extern "C" int solweig_patch_sums(const uint32_t* masks, int64_t pixels, int patches, const float* weights,
                                  int ncols, float* out, void* work, int64_t work_bytes, void* stream) {
    SOLWEIG_CHECK_ARG(masks && weights && out && work && pixels > 0, "solweig_patch_sums: null argument");
    SOLWEIG_CHECK_ARG(patches > 0 && patches <= kK, "solweig_patch_sums: patches %d outside 1..%d", patches, kK);
    SOLWEIG_CHECK_ARG(ncols > 0 && ncols <= 256, "solweig_patch_sums: ncols %d outside 1..256", ncols);
    const int nb = (ncols + 15) / 16 * 16;
    const long long need = 2LL * 2 * nb * kK + 16;
    SOLWEIG_CHECK_ARG(work_bytes >= need, "solweig_patch_sums: work buffer of %lld bytes, need %lld",
                      (long long)work_bytes, need);
    SOLWEIG_CHECK_ARG(((uintptr_t)work & 15) == 0, "solweig_patch_sums: work buffer not 16-byte aligned");
    cudaStream_t st = as_stream(stream);
    __nv_bfloat16* b = reinterpret_cast<__nv_bfloat16*>(work);
    int* err = reinterpret_cast<int*>(static_cast<char*>(work) + 2LL * 2 * nb * kK);
    cudaMemsetAsync(err, 0, sizeof(int), st);
    split_bf16_kernel<<<blocks_for((long long)nb * kK, 256), 256, 0, st>>>(weights, ncols, nb, patches, b);
    SOLWEIG_CHECK_LAUNCH("split_bf16_kernel");
    return launch_gemm(masks, pixels, patches, b, ncols, nb, out, err, st);
}

namespace {

constexpr int kDayStages = 5;  // shadow, GVF, weights + tables, contraction, radiation

// Parts of a day: kDaySweep runs the sweep stage (ray exits, ceilings and the
// shadow sweep) of hours [h0, h1) -- the part that starts at hour 0 also
// builds the day's dilated height planes; kDayRest runs everything after it
// (GVF to radiation) over all hours; kDayAll both.
enum DayPart { kDaySweep = 0, kDayRest = 1, kDayAll = 2 };

int day_batched_impl(const SolweigScene* scene, const SolweigSkyLayout* layout, const SolweigHour* hours,
                     int nhours, const SolweigState* state, const SolweigOutputs* base, int64_t hour_stride,
                     const int32_t* gvf_dxdy, int first_steps, int second_steps, void* work,
                     int64_t work_bytes, void* stream, cudaEvent_t* ev, const SolweigDayConfig* cfg_in,
                     int part = kDayAll, int h0 = 0, int h1 = -1) {
    SolweigDayConfig cfg{16, 16, 8, 256, 0, 1, 0, 0};
    if (cfg_in) cfg = *cfg_in;
    SOLWEIG_CHECK_ARG(cfg.shadow_bx > 0 && cfg.shadow_by > 0 && cfg.shadow_bx * cfg.shadow_by <= 256 &&
                          (cfg.shadow_bx * cfg.shadow_by) % 32 == 0,
                      "solweig_day_batched: shadow block %dx%d (at most 256 threads, a multiple of 32)",
                      cfg.shadow_bx, cfg.shadow_by);
    SOLWEIG_CHECK_ARG(cfg.gvf_rows == 4 || cfg.gvf_rows == 8 || cfg.gvf_rows == 16,
                      "solweig_day_batched: gvf_rows must be 4, 8 or 16");
    SOLWEIG_CHECK_ARG(cfg.rad_threads == 128 || cfg.rad_threads == 256,
                      "solweig_day_batched: rad_threads must be 128 or 256");
    SOLWEIG_CHECK_ARG(cfg.gemm_ctas_per_sm >= 0 && cfg.gemm_ctas_per_sm <= 2,
                      "solweig_day_batched: gemm_ctas_per_sm must be 0 (auto), 1 or 2");
    SOLWEIG_CHECK_ARG(cfg.gvf_hours == 0 || cfg.gvf_hours == 1, "solweig_day_batched: gvf_hours must be 0 or 1");
    SOLWEIG_CHECK_ARG(cfg.no_ceiling == 0 || cfg.no_ceiling == 1, "solweig_day_batched: no_ceiling must be 0 or 1");
    SOLWEIG_CHECK_ARG(cfg.sweep_window >= 0 && cfg.sweep_window <= 2,
                      "solweig_day_batched: sweep_window must be 0, 1 or 2");
    SOLWEIG_CHECK_ARG(scene && layout && hours && base && work, "solweig_day_batched: null argument");
    const SolweigScene& S = *scene;
    SOLWEIG_CHECK_ARG(S.rows > 0 && S.cols > 0, "solweig_day_batched: bad scene shape %dx%d", S.rows, S.cols);
    SOLWEIG_CHECK_ARG(nhours > 0 && nhours <= kMaxDayHours, "solweig_day_batched: nhours %d outside 1..%d",
                      nhours, kMaxDayHours);
    SOLWEIG_CHECK_ARG(S.patches == 153 || S.patches == 145,
                      "solweig_day_batched: sky layout with %d patches (145 or 153 supported)", S.patches);
    SOLWEIG_CHECK_ARG(!(base->keast || base->ksouth || base->kwest || base->knorth || base->least ||
                        base->lsouth || base->lwest || base->lnorth),
                      "solweig_day_batched: cardinal planes are not produced by the batched form");
    SOLWEIG_CHECK_ARG(gvf_dxdy && second_steps >= 1 && second_steps <= SOLWEIG_GVF_MAX_STEPS &&
                          first_steps >= 1 && first_steps <= second_steps,
                      "solweig_day_batched: GVF steps first=%d second=%d", first_steps, second_steps);
    const long long px = (long long)S.rows * S.cols;
    const DayWork w = day_work_layout(px, nhours, S.has_water != 0);
    SOLWEIG_CHECK_ARG(work_bytes >= w.total, "solweig_day_batched: work buffer of %lld bytes, need %lld",
                      (long long)work_bytes, w.total);
    SOLWEIG_CHECK_ARG(((uintptr_t)work & 255) == 0, "solweig_day_batched: work buffer not 256-byte aligned");
    char* wb = static_cast<char*>(work);
    float4* quads = reinterpret_cast<float4*>(wb + w.quads);
    float* lup_first = S.has_water ? reinterpret_cast<float*>(wb + w.lup_first) : nullptr;
    float* gvf = reinterpret_cast<float*>(wb + w.gvf);
    float* nosh = reinterpret_cast<float*>(wb + w.nosh);
    float* sums = reinterpret_cast<float*>(wb + w.sums);
    float* wf32 = reinterpret_cast<float*>(wb + w.wf32);
    __nv_bfloat16* bw = reinterpret_cast<__nv_bfloat16*>(wb + w.bw);
    DayTable* tables = reinterpret_cast<DayTable*>(wb + w.tables);
    int* err = reinterpret_cast<int*>(wb + w.error);
    float* tmax = reinterpret_cast<float*>(wb + w.tilemax);
    // the window sweep: packed geometry (16-byte aligned for the tensor map), no water
    const bool window = cfg.sweep_window != 0 && S.geo32 && !S.has_water && ((uintptr_t)S.geo32 & 15) == 0;
    cudaStream_t st = as_stream(stream);

    DayGvfArgs ga{first_steps, second_steps, second_steps - 1};
    const int halo = ga.halo;
    for (int i = 0; i < 2 * SOLWEIG_GVF_DIRECTIONS * second_steps; ++i)
        SOLWEIG_CHECK_ARG(gvf_dxdy[i] >= -halo && gvf_dxdy[i] <= halo,
                          "solweig_day_batched: GVF offset %d outside the halo %d", gvf_dxdy[i], halo);
    const int pitch = 32 + 2 * halo;
    SOLWEIG_CHECK_ARG(sizeof(float4) * (size_t)pitch * (8 + 2 * halo) <= 227 * 1024,
                      "solweig_day_batched: GVF halo %d too large", halo);

    if (h1 < 0) h1 = nhours;
    SOLWEIG_CHECK_ARG(part == kDaySweep || part == kDayRest || part == kDayAll,
                      "solweig_day_batched: unknown part %d", part);
    SOLWEIG_CHECK_ARG(0 <= h0 && h0 < h1 && h1 <= nhours, "solweig_day_batched: hours [%d, %d) outside [0, %d)", h0,
                      h1, nhours);
    if (part == kDayAll) {
        if (ev) cudaEventRecord(ev[0], st);
        int rc = day_batched_impl(scene, layout, hours, nhours, state, base, hour_stride, gvf_dxdy, first_steps,
                                  second_steps, work, work_bytes, stream, nullptr, &cfg, kDaySweep, 0, nhours);
        if (rc) return rc;
        if (ev) cudaEventRecord(ev[1], st);
        return day_batched_impl(scene, layout, hours, nhours, state, base, hour_stride, gvf_dxdy, first_steps,
                                second_steps, work, work_bytes, stream, ev, &cfg, kDayRest, 0, nhours);
    }
    if (part == kDaySweep) {
        const int nh = h1 - h0;
        // The ceiling planes (8 B per pixel-hour: ceiling and window maximum)
        // live in the GVF region (12 B
        // per pixel-hour) and the four dilated height planes (16 B per pixel)
        // in the patch-sum region (at least 16 B per pixel): both are consumed
        // by the sweep before the GVF kernels and the contraction write those
        // regions.
        float2* ceiling = cfg.no_ceiling ? nullptr : reinterpret_cast<float2*>(gvf);
        float* dil = sums;
        if (h0 == 0) {
            cudaMemsetAsync(err, 0, sizeof(int), st);  // the day's error flag
            if (window) {  // 16 x 16 tile maxima of the heights, for the warp vote
                const long long ntiles = (long long)sweep_tiles_along(S.rows) * sweep_tiles_along(S.cols);
                sweep_tile_max_kernel<<<blocks_for(ntiles, 8), 256, 0, st>>>(S, tmax);
                SOLWEIG_CHECK_LAUNCH("sweep_tile_max_kernel");
            }
        }
        if (ceiling && h0 == 0) {
            dim3 dgrid(blocks_for(S.cols, kDilTile), blocks_for(S.rows, kDilTile));
            if (S.geo32) ceiling_dilate_kernel<true><<<dgrid, dim3(32, 8), 0, st>>>(S, dil);
            else ceiling_dilate_kernel<false><<<dgrid, dim3(32, 8), 0, st>>>(S, dil);
            SOLWEIG_CHECK_LAUNCH("ceiling_dilate_kernel");
        }
        if (ceiling) {
            dim3 grid(blocks_for((long long)S.rows + S.cols, kCeilLanes), 1, nh);
            day_ray_ceiling_kernel<<<grid, dim3(kCeilLanes, kCeilWarps), 0, st>>>(S, hours + h0, dil,
                                                                                  ceiling + h0 * px);
            SOLWEIG_CHECK_LAUNCH("day_ray_ceiling_kernel");
        }
        // first-outside steps of every row and column per hour (4 B each), in
        // the GVF region after the ceiling planes (4 B per pixel-hour left; a
        // raster one pixel wide spills a few bytes into the next region, free
        // until the GVF stage)
        int* exits = reinterpret_cast<int*>(wb + w.gvf + 8LL * px * nhours) + (long long)h0 * (S.rows + S.cols);
        // then the hours' step records (16 B per step, at most max(rows, cols) + 2
        // steps per hour), when they fit before the end of the GVF region
        const long long rec_at = (w.gvf + 8LL * px * nhours + 4LL * (S.rows + S.cols) * nhours + 15) & ~15LL;
        const int kmax = (S.rows > S.cols ? S.rows : S.cols) + 2;
        longlong2* rec = nullptr;
        if (rec_at + 16LL * kmax * nhours <= w.gvf + 12LL * px * nhours)
            rec = reinterpret_cast<longlong2*>(wb + rec_at) + (long long)h0 * kmax;
        day_ray_exits_kernel<<<nh, 1024, 0, st>>>(S, hours + h0, exits, rec, kmax, err);
        SOLWEIG_CHECK_LAUNCH("day_ray_exits_kernel");
        if (window) {
            const int win = cfg.sweep_window == 2 ? 40 : 48;
            CUtensorMap map;
            const int rc = sweep_geo_map(S, win, &map);
            if (rc) return rc;
            dim3 grid(blocks_for(S.cols, kSwTile), blocks_for(S.rows, kSwTile), nh);
            const float2* ceil0 = ceiling ? ceiling + h0 * px : nullptr;
            if (win == 40) {
                set_smem_attr((const void*)day_sweep_tma_kernel<40>, sweep_smem_bytes<40>());
                day_sweep_tma_kernel<40><<<grid, kSwThreads, sweep_smem_bytes<40>(), st>>>(
                    map, S, hours + h0, quads + h0 * px, ceil0, exits, tmax, err);
            } else {
                set_smem_attr((const void*)day_sweep_tma_kernel<48>, sweep_smem_bytes<48>());
                day_sweep_tma_kernel<48><<<grid, kSwThreads, sweep_smem_bytes<48>(), st>>>(
                    map, S, hours + h0, quads + h0 * px, ceil0, exits, tmax, err);
            }
            SOLWEIG_CHECK_LAUNCH("day_sweep_tma_kernel");
            return SOLWEIG_OK;
        }
        dim3 grid(blocks_for(S.cols, cfg.shadow_bx), blocks_for(S.rows, cfg.shadow_by), nh);
        if (rec && S.geo32)
            day_shadow_kernel<true><<<grid, dim3(cfg.shadow_bx, cfg.shadow_by), 0, st>>>(
                S, hours + h0, quads + h0 * px, lup_first ? lup_first + h0 * px : nullptr,
                ceiling ? ceiling + h0 * px : nullptr, exits, rec, kmax);
        else
            day_shadow_kernel<false><<<grid, dim3(cfg.shadow_bx, cfg.shadow_by), 0, st>>>(
                S, hours + h0, quads + h0 * px, lup_first ? lup_first + h0 * px : nullptr,
                ceiling ? ceiling + h0 * px : nullptr, exits, nullptr, 0);
        SOLWEIG_CHECK_LAUNCH("day_shadow_kernel");
        return SOLWEIG_OK;
    }
    // kDayRest (the error flag was cleared by the sweep part of hour 0)
    cudaMemsetAsync(nosh, 0, 4 * px, st);
    if (first_steps == 1 && second_steps == 22) {
        GvfTable<22> tab;
        fill_day_table(tab, gvf_dxdy, 22, pitch);
        const bool hv = cfg.gvf_hours == 1 && !S.has_water;
        if (!hv) {
            launch_day_gvf<1, 22, 22>(cfg.gvf_rows, S, hours, nhours, ga, tab, quads, lup_first, gvf, nosh, st);
        } else {
            const size_t smem = hv_smem_bytes();
            set_smem_attr((const void*)day_gvf_hv_kernel, smem);
            dim3 grid(blocks_for(S.cols, kHvTile), blocks_for(S.rows, kHvTile));
            day_gvf_hv_kernel<<<grid, dim3(kHvTile, kHvTile), smem, st>>>(S, hours, nhours, tab, quads, gvf, nosh);
            SOLWEIG_CHECK_LAUNCH("day_gvf_hv_kernel");
        }
    } else {
        GvfTable<SOLWEIG_GVF_MAX_STEPS> tab;
        fill_day_table(tab, gvf_dxdy, second_steps, pitch);
        launch_day_gvf<0, 0, SOLWEIG_GVF_MAX_STEPS>(cfg.gvf_rows, S, hours, nhours, ga, tab, quads, lup_first, gvf,
                                                    nosh, st);
    }
    SOLWEIG_CHECK_LAUNCH("day_gvf_kernel");
    if (ev) cudaEventRecord(ev[2], st);

    const int ncols = 2 * nhours;
    const int nb = (ncols + 15) / 16 * 16;
    day_weights_kernel<<<blocks_for((long long)ncols * kK, 256), 256, 0, st>>>(layout, hours, nhours, wf32);
    SOLWEIG_CHECK_LAUNCH("day_weights_kernel");
    // sky weights, then the vegetation weights prescaled by the diffuse
    // transmissivity of vegetation (0.03, src/svf.py:117-131): one set of sums
    split_bf16_kernel<<<blocks_for((long long)nb * kK, 256), 256, 0, st>>>(wf32, ncols, nb, S.patches, bw);
    split_bf16_kernel<<<blocks_for((long long)nb * kK, 256), 256, 0, st>>>(wf32, ncols, nb, S.patches,
                                                                           bw + 2LL * nb * kK, 0.03f);
    SOLWEIG_CHECK_LAUNCH("split_bf16_kernel");
    day_tables_kernel<<<nhours, kK, 0, st>>>(layout, hours, tables);
    SOLWEIG_CHECK_LAUNCH("day_tables_kernel");
    if (ev) cudaEventRecord(ev[3], st);
    int rc = launch_gemm(S.masks, px, S.patches, bw, ncols, nb, sums, err, st, cfg.gemm_ctas_per_sm, true);
    if (rc) return rc;
    if (ev) cudaEventRecord(ev[4], st);

    DayRadArgs ra{};
    ra.layout = layout;
    ra.hours = hours;
    ra.nhours = nhours;
    ra.tables = tables;
    ra.gvf = gvf;
    ra.nosh = nosh;
    ra.sums = sums;
    ra.ncols = ncols;
    if (state) ra.state = *state;
    ra.out = *base;
    ra.hour_stride = hour_stride;
    const unsigned blocks = blocks_for(px, cfg.rad_threads);
    if (cfg.rad_threads == 128) {
        if (S.patches == 153) day_radiation_kernel<2, 128><<<blocks, 128, 0, st>>>(S, ra);
        else day_radiation_kernel<1, 128><<<blocks, 128, 0, st>>>(S, ra);
    } else {
        if (S.patches == 153) day_radiation_kernel<2, 256><<<blocks, 256, 0, st>>>(S, ra);
        else day_radiation_kernel<1, 256><<<blocks, 256, 0, st>>>(S, ra);
    }
    SOLWEIG_CHECK_LAUNCH("day_radiation_kernel");
    if (ev) cudaEventRecord(ev[5], st);
    return SOLWEIG_OK;
}

}  // namespace

extern "C" int solweig_day_batched(const SolweigScene* scene, const SolweigSkyLayout* layout,
                                   const SolweigHour* hours, int nhours, const SolweigState* state,
                                   const SolweigOutputs* base, int64_t hour_stride, const int32_t* gvf_dxdy,
                                   int first_steps, int second_steps, void* work, int64_t work_bytes,
                                   void* stream) {
    return day_batched_impl(scene, layout, hours, nhours, state, base, hour_stride, gvf_dxdy, first_steps,
                            second_steps, work, work_bytes, stream, nullptr, nullptr);
}

extern "C" int solweig_day_batched_ex(const SolweigScene* scene, const SolweigSkyLayout* layout,
                                      const SolweigHour* hours, int nhours, const SolweigState* state,
                                      const SolweigOutputs* base, int64_t hour_stride, const int32_t* gvf_dxdy,
                                      int first_steps, int second_steps, void* work, int64_t work_bytes,
                                      const SolweigDayConfig* config, void* stream) {
    return day_batched_impl(scene, layout, hours, nhours, state, base, hour_stride, gvf_dxdy, first_steps,
                            second_steps, work, work_bytes, stream, nullptr, config);
}

// One part of solweig_day_batched_ex (no counterpart in the reference): with
// part 0 the sweep stage of hours [hour_begin, hour_end), with part 1 the
// rest of the day over all hours.  Calling part 0 over consecutive ranges
// covering [0, nhours) in order and then part 1 on one stream gives the
// results of solweig_day_batched_ex; the host can plan later hours while
// the earlier ranges run.
extern "C" int solweig_day_batched_part(const SolweigScene* scene, const SolweigSkyLayout* layout,
                                        const SolweigHour* hours, int nhours, const SolweigState* state,
                                        const SolweigOutputs* base, int64_t hour_stride, const int32_t* gvf_dxdy,
                                        int first_steps, int second_steps, void* work, int64_t work_bytes,
                                        const SolweigDayConfig* config, int part, int hour_begin, int hour_end,
                                        void* stream) {
    SOLWEIG_CHECK_ARG(part == 0 || part == 1, "solweig_day_batched_part: part must be 0 or 1");
    if (part == 1) {
        hour_begin = 0;
        hour_end = nhours;
    }
    return day_batched_impl(scene, layout, hours, nhours, state, base, hour_stride, gvf_dxdy, first_steps,
                            second_steps, work, work_bytes, stream, nullptr, config,
                            part == 0 ? kDaySweep : kDayRest, hour_begin, hour_end);
}

extern "C" int solweig_day_batched_timed(const SolweigScene* scene, const SolweigSkyLayout* layout,
                                         const SolweigHour* hours, int nhours, const SolweigState* state,
                                         const SolweigOutputs* base, int64_t hour_stride,
                                         const int32_t* gvf_dxdy, int first_steps, int second_steps, void* work,
                                         int64_t work_bytes, const SolweigDayConfig* config, void* stream,
                                         float* stage_ms) {
    SOLWEIG_CHECK_ARG(stage_ms, "solweig_day_batched_timed: null stage_ms");
    cudaEvent_t ev[kDayStages + 1];
    for (int i = 0; i <= kDayStages; ++i) {
        const cudaError_t e = cudaEventCreate(&ev[i]);
        if (e != cudaSuccess) {
            for (int j = 0; j < i; ++j) cudaEventDestroy(ev[j]);
            set_error("solweig_day_batched_timed: cudaEventCreate: %s", cudaGetErrorString(e));
            return SOLWEIG_ERR_CUDA;
        }
    }
    int rc = day_batched_impl(scene, layout, hours, nhours, state, base, hour_stride, gvf_dxdy, first_steps,
                              second_steps, work, work_bytes, stream, ev, config);
    if (rc == SOLWEIG_OK) {
        const cudaError_t e = cudaEventSynchronize(ev[kDayStages]);
        if (e != cudaSuccess) {
            set_error("solweig_day_batched_timed: %s", cudaGetErrorString(e));
            rc = SOLWEIG_ERR_CUDA;
        } else {
            for (int i = 0; i < kDayStages; ++i) cudaEventElapsedTime(&stage_ms[i], ev[i], ev[i + 1]);
        }
    }
    for (int i = 0; i <= kDayStages; ++i) cudaEventDestroy(ev[i]);
    return rc;
}

// Device error flag of the last batched day run in `work` (0 = none, 1 = a
// tensor-core wait timed out); copied to *out on `stream`.
extern "C" int solweig_day_batched_error(const void* work, int rows, int cols, int nhours, int has_water,
                                         int* out_device, void* stream) {
    SOLWEIG_CHECK_ARG(work && out_device, "solweig_day_batched_error: null argument");
    const DayWork w = day_work_layout((long long)rows * cols, nhours, has_water != 0);
    cudaMemcpyAsync(out_device, static_cast<const char*>(work) + w.error, sizeof(int), cudaMemcpyDeviceToDevice,
                    as_stream(stream));
    return SOLWEIG_OK;
}
