// Static scene preparation on the device (src/series.py:252-349).
//
// solweig_scene_build: per-pixel derivations from the input rasters
//   (DSM raise, canopy / trunk-zone tops, bush, buildings mask, land-cover
//   maps through the class table of src/landcoverclasses_2016a.txt);
// solweig_scene_finalize: fields derived from the SVF planes after their
//   float32 round trip (src/series.py:337-349) plus the per-direction wall
//   face bits used by the ground view factor.
#include "common.cuh"

namespace solweig {

struct BuildParams {
    long long n;
    double raise_dsm, raise_dem;
    int landcover;
    // class table rows: code, albedo, emissivity, TgK, Tstart, TmaxLST
    int nclasses;
    double classes[16][6];
    double def_alb, def_emis, def_tgk, def_tstart, def_tmaxlst;
};

__global__ void __launch_bounds__(256) scene_build_kernel(
    const double* __restrict__ dsm_in, const double* __restrict__ trees_in,
    const double* __restrict__ dem_in, const double* __restrict__ lc_in, BuildParams prm,
    double* __restrict__ dsm, double* __restrict__ vegdem, double* __restrict__ vegdem2,
    uint8_t* __restrict__ flags, float* __restrict__ alb, float* __restrict__ emis,
    float* __restrict__ tgk, float* __restrict__ tstart, float* __restrict__ tmaxlst,
    float* __restrict__ lc_out) {
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= prm.n) return;
    double a = dsm_in[p];
    if (prm.raise_dsm != 0.0) a = a + prm.raise_dsm;
    double dem = dem_in[p];
    if (prm.raise_dem != 0.0) dem = dem + prm.raise_dem;
    double t1 = trees_in[p];
    if (t1 < 0.0) t1 = 0.0;
    double top = t1 + a;
    if (top == a) top = 0.0;
    double bot = t1 * 0.25 + a;
    if (bot == a) bot = 0.0;
    const double bush = (bot * top == 0.0 ? 1.0 : 0.0) * top;
    double b = a - dem;
    if (b < 2.0) b = 1.0;
    else if (b >= 2.0) b = 0.0;
    dsm[p] = a;
    vegdem[p] = top;
    vegdem2[p] = bot;
    double code = 0.0;
    double al = prm.def_alb, em = prm.def_emis, tk = prm.def_tgk, ts = prm.def_tstart,
           tm = prm.def_tmaxlst;
    if (prm.landcover) {
        const double src = lc_in[p];
        double r = rint(src);
        // isclose(src, r) with numpy's default tolerances
        const bool close = fabs(src - r) <= 1e-8 + 1e-5 * fabs(r);
        if (!isfinite(src) || !close || r < 1.0 || r > 7.0) r = 6.0;
        if (r == 3.0 || r == 4.0) r = 5.0;
        code = (double)(float)r;
        for (int k = 0; k < prm.nclasses; ++k)
            if (prm.classes[k][0] == code) {
                al = prm.classes[k][1];
                em = prm.classes[k][2];
                tk = prm.classes[k][3];
                ts = prm.classes[k][4];
                tm = prm.classes[k][5];
            }
    }
    alb[p] = (float)al;
    emis[p] = (float)em;
    tgk[p] = (float)tk;
    tstart[p] = (float)ts;
    tmaxlst[p] = (float)tm;
    if (lc_out) lc_out[p] = (float)code;
    flags[p] = (uint8_t)((b == 1.0 ? 1 : 0) | (bush > 1.0 ? 2 : 0) | (code == 3.0 ? 4 : 0));
}

struct FinalizeParams {
    long long n;
    double trans;
    double face_low[SOLWEIG_GVF_DIRECTIONS], face_high[SOLWEIG_GVF_DIRECTIONS];
    int face_middle[SOLWEIG_GVF_DIRECTIONS];
};

// planes: the 16 float64 planes of solweig_svf in its reduce order
// (0 all, 1 E, 2 S, 3 W, 4 N for sh; 5..9 veg; 10..14 vb; 15 total).
__global__ void __launch_bounds__(256) scene_finalize_kernel(
    const double* __restrict__ planes, const double* __restrict__ walls,
    const double* __restrict__ aspect_rad, FinalizeParams prm, float* __restrict__ svf32,
    float* __restrict__ svfbuveg, double* __restrict__ svfalfa, double* __restrict__ tan_asvf,
    uint32_t* __restrict__ gvf_face) {
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= prm.n) return;
    const long long n = prm.n;
    // float32 round trip of the 15 SVF planes
    double v[15];
#pragma unroll
    for (int i = 0; i < 15; ++i) {
        const float f = (float)planes[(long long)i * n + p];
        v[i] = (double)f;
        if (svf32) svf32[(long long)i * n + p] = f;
    }
    const double svf = v[0], svfveg = v[5];
    svfbuveg[p] = (float)(svf - (1.0 - svfveg) * (1.0 - prm.trans));
    tan_asvf[p] = tan(acos(sqrt(svf)));
    double tmp = svf + svfveg - 1.0;
    if (tmp < 0.0) tmp = 0.0;
    svfalfa[p] = asin(exp(log(1.0 - tmp) / 2.0));
    const double wall = walls[p];
    const double wallbol = wall > 0.0 ? 1.0 : 0.0;
    const double asp = aspect_rad[p];
    uint32_t mask = 0;
    for (int j = 0; j < SOLWEIG_GVF_DIRECTIONS; ++j) {
        const double lo = prm.face_low[j], hi = prm.face_high[j];
        const double facesh = prm.face_middle[j] ? (double)(asp < lo || asp >= hi) - wallbol + 1.0
                                                 : 1.0 - (double)(asp > lo || asp <= hi);
        if (facesh == 0.0) mask |= 1u << j;
    }
    gvf_face[p] = mask;
}

}  // namespace solweig

using namespace solweig;

extern "C" int solweig_scene_build(const double* dsm_in, const double* trees_in, const double* dem_in,
                                   const double* landcover_in, int64_t pixels, double raise_dsm,
                                   double raise_dem, const double* classes, int nclasses,
                                   const double* defaults /* alb, emis, TgK, Tstart, TmaxLST */,
                                   double* dsm, double* vegdem, double* vegdem2, uint8_t* flags,
                                   float* alb, float* emis, float* tgk, float* tstart,
                                   float* tmaxlst, float* lc_out, void* stream) {
    SOLWEIG_CHECK_ARG(dsm_in && trees_in && dem_in && defaults && dsm && vegdem && vegdem2 && flags &&
                          alb && emis && tgk && tstart && tmaxlst && pixels > 0,
                      "solweig_scene_build: bad arguments");
    SOLWEIG_CHECK_ARG(!landcover_in || (classes && nclasses > 0 && nclasses <= 16),
                      "solweig_scene_build: land cover needs 1..16 classes");
    BuildParams prm{};
    prm.n = pixels;
    prm.raise_dsm = raise_dsm;
    prm.raise_dem = raise_dem;
    prm.landcover = landcover_in != nullptr;
    prm.nclasses = landcover_in ? nclasses : 0;
    for (int k = 0; k < prm.nclasses; ++k)
        for (int j = 0; j < 6; ++j) prm.classes[k][j] = classes[6 * k + j];
    prm.def_alb = defaults[0];
    prm.def_emis = defaults[1];
    prm.def_tgk = defaults[2];
    prm.def_tstart = defaults[3];
    prm.def_tmaxlst = defaults[4];
    scene_build_kernel<<<blocks_for(pixels, 256), 256, 0, as_stream(stream)>>>(
        dsm_in, trees_in, dem_in, landcover_in, prm, dsm, vegdem, vegdem2, flags, alb, emis, tgk,
        tstart, tmaxlst, lc_out);
    SOLWEIG_CHECK_LAUNCH("scene_build_kernel");
    return SOLWEIG_OK;
}

extern "C" int solweig_scene_finalize(const double* planes, const double* walls,
                                      const double* aspect_rad, int64_t pixels, double transmissivity,
                                      const double* face_low, const double* face_high,
                                      const int32_t* face_middle, float* svf32, float* svfbuveg,
                                      double* svfalfa, double* tan_asvf, uint32_t* gvf_face,
                                      void* stream) {
    SOLWEIG_CHECK_ARG(planes && walls && aspect_rad && face_low && face_high && face_middle &&
                          svfbuveg && svfalfa && tan_asvf && gvf_face && pixels > 0,
                      "solweig_scene_finalize: bad arguments");
    FinalizeParams prm{};
    prm.n = pixels;
    prm.trans = transmissivity;
    for (int j = 0; j < SOLWEIG_GVF_DIRECTIONS; ++j) {
        prm.face_low[j] = face_low[j];
        prm.face_high[j] = face_high[j];
        prm.face_middle[j] = face_middle[j];
    }
    scene_finalize_kernel<<<blocks_for(pixels, 256), 256, 0, as_stream(stream)>>>(
        planes, walls, aspect_rad, prm, svf32, svfbuveg, svfalfa, tan_asvf, gvf_face);
    SOLWEIG_CHECK_LAUNCH("scene_finalize_kernel");
    return SOLWEIG_OK;
}
