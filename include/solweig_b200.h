/*
 * solweig_b200.h -- C ABI of libsolweig_b200.so, the sm_100a SOLWEIG engine.
 *
 * Every entry point takes device pointers that the caller allocated, plain
 * sizes and a CUDA stream (as void*; NULL = default stream), launches its
 * kernels on that stream, performs no hidden synchronisation and returns an
 * int status (SOLWEIG_OK = 0).  On failure solweig_last_error() returns a
 * message for the calling thread.  Nothing here allocates device memory.
 *
 * Raster layout: row-major [rows][cols]; "rows" is axis 0 of the reference's
 * numpy arrays.  Per-patch visibility is bit-packed: two planes (S, V) of
 * SOLWEIG_MASK_WORDS uint32 words per pixel, stored plane-major as
 * masks[(plane * SOLWEIG_MASK_WORDS + word) * pixels + pixel]; bit k of word
 * w is patch 32*w + k.  S = no building in that direction (the reference's
 * shmat == 1), V = vegetation seen (vegshmat == 0 or vbshvegshmat == 0).
 * The four states of a (pixel, patch) pair are then
 *   sky  = S & ~V,  vegetation = S & V,  building = ~S & ~V,
 *   building behind vegetation = ~S & V.
 *
 * Reference interfaces replaced (paths relative to the reference root):
 *   solweig_wall_heights      src/walls.py:59-69, src/kernels/geometry.cu:15-34
 *   solweig_wall_aspect       src/walls.py:83-121, src/kernels/geometry.cu:36-63
 *   solweig_wall_segments_burn, solweig_geometry_walls
 *                             src/walls.py:270-332 (calculate_geometry_walls)
 *   solweig_shadow            src/model.py:689-708 (cast_shadow),
 *                             src/kernels/geometry.cu:185-253
 *   solweig_svf               src/svf.py:81-114, src/kernels/geometry.cu:77-159
 *   solweig_svf_unpack        src/svf.py:113-114 (the three [rows,cols,P] cubes)
 *   solweig_diffsh            src/svf.py:117-131, src/kernels/geometry.cu:161-172
 *   solweig_gvf               src/model.py:569-622, src/kernels/gvf.cu:79-292
 *   solweig_step(_shadow,_radiation)
 *                             src/model.py:15-256 (Solweig_2022a_calc, device part)
 *   solweig_step64            the same step under the float64 switch (run.py:27,
 *                             src/runtime.py:43-49)
 *   solweig_day               src/series.py:445-491 (the hour loop of _run_day)
 *   solweig_day_batched       src/series.py:445-491 (same loop, batched form)
 *   solweig_scene_build/finalize src/series.py:252-349 (_prepare_spatial, per pixel)
 *   solweig_utci              src/utci.py:6-33, src/kernels/utci.cu
 */
#ifndef SOLWEIG_B200_H
#define SOLWEIG_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SOLWEIG_OK 0
#define SOLWEIG_ERR_INVALID 1
#define SOLWEIG_ERR_CUDA 2
#define SOLWEIG_ERR_TIMEOUT 3

#define SOLWEIG_MAX_PATCHES 160
#define SOLWEIG_MASK_WORDS 5
#define SOLWEIG_MAX_BANDS 8
#define SOLWEIG_GVF_DIRECTIONS 18
#define SOLWEIG_GVF_MAX_STEPS 64

/* Static per-scene device arrays (all [rows*cols] unless noted). */
typedef struct SolweigScene {
    int32_t rows, cols;
    double scale;             /* 1 / pixel size */
    /* geometry, float64 (exact comparisons in the shadow sweep) */
    const double* dsm;        /* building DSM raised to >= 0 */
    const double* vegdem;     /* canopy top (0 where no vegetation) */
    const double* vegdem2;    /* trunk-zone top (0 where none) */
    const double* walls;      /* wall height, m (0 = no wall) */
    const double* aspect;     /* wall aspect, radians */
    const uint8_t* flags;     /* bit0 ground (buildings==1), bit1 bush>1, bit2 water (lc==3) */
    /* land cover and radiation statics, float32 */
    const float* alb;         /* ground albedo */
    const float* emis;        /* ground emissivity */
    const float* tgk;         /* TgK */
    const float* tstart;      /* Tstart */
    const float* tmaxlst;     /* TmaxLST */
    const float* svfbuveg;    /* svf - (1 - svfveg)(1 - transVeg) */
    const double* svfalfa;    /* asin(exp(log(1 - max(svf + svfveg - 1, 0)) / 2)) */
    const double* tan_asvf;   /* tan(acos(sqrt(svf))) */
    const uint32_t* masks;    /* SOLWEIG_MASK_WORDS * 2 planes, see above */
    const float* veg_sums;    /* [4][pixels]: sum over V of omega*cos, omega*sin; over
                                 obstructed (~sky) of omega*cos, omega*sin */
    const uint8_t* sky_band_counts; /* [nbands][pixels]: sky patches per band */
    const uint32_t* gvf_face;  /* bit j: wall face turned away from GVF direction j (facesh==0) */
    /* isotropic / box variants read these directional SVFs (may be NULL otherwise) */
    const float* svf_dir;     /* [12][pixels]: E,S,W,N x (svf, svfveg, svfaveg) */
    int32_t patches;          /* number of sky patches (153 for option 2) */
    int32_t nbands;
    int32_t landcover;        /* 1 = land-cover maps in use (enables Tg clamp / water) */
    int32_t has_water;        /* any flags bit2 set */
    double hmax;              /* max over the raster of dsm, vegdem, vegdem2 */
    /* optional: float4 (dsm, vegdem, vegdem2, 0) per pixel, set only when every
       value of the three rasters is exactly representable in float32 (the
       hourly shadow sweep then loads one 16-byte sample per step); NULL otherwise */
    const void* geo32;
    /* optional statics of the batched day's hour-vectorized GVF (1 m walk, no
       water), from solweig_gvf_statics: walk-length codes [4][pixels] and the
       albedo-without-shadow GVF [pixels]; NULL: the day walks them itself */
    const uint32_t* gvf_hits;
    const float* gvf_nosh;
} SolweigScene;

/* Per-patch constants of the sky-vault layout (host arrays, copied per call). */
typedef struct SolweigSkyLayout {
    int32_t patches, nbands;
    int32_t band_of_patch[SOLWEIG_MAX_PATCHES];
    float omega[SOLWEIG_MAX_PATCHES];       /* steradian */
    float cos_alt[SOLWEIG_MAX_PATCHES];
    float sin_alt[SOLWEIG_MAX_PATCHES];
    float band_omega[SOLWEIG_MAX_BANDS];
    float band_cos[SOLWEIG_MAX_BANDS];
    float band_sin[SOLWEIG_MAX_BANDS];
    double sunlit_below[SOLWEIG_MAX_PATCHES]; /* x < t  <=> atan(x)*180/pi < patch altitude */
    double shaded_above[SOLWEIG_MAX_PATCHES]; /* x > t  <=> atan(x)*180/pi > patch altitude */
    float cardinal[4][SOLWEIG_MAX_PATCHES];  /* E,S,W,N longwave direction cosines (0 = off) */
} SolweigSkyLayout;

/* One hour: FP64 host scalars and the device ray table of the sun. */
typedef struct SolweigHour {
    int32_t daytime;          /* altitude > 0 */
    double altitude, azimuth; /* degrees */
    double zen;               /* radians */
    double ta, rh, ws;        /* deg C, %, m/s */
    double rad_g, rad_d, rad_i;
    double psi;               /* 1 - vegetation transmissivity */
    double cos_alt, sin_alt;  /* of the solar altitude */
    double tan_zen;
    double esky;              /* after the CI < 0.95 blend */
    double ci_tgg;            /* CI_TgG */
    double tg_phase;          /* sin(...) factor of Tg for ground (per pixel TmaxLST => see tgk) */
    double altmax, dectime_frac, snup;
    double tgwall;            /* wall temperature amplitude after CI scaling and clamp */
    double twater;
    int32_t firstdaytime;     /* TsWaveDelay flags */
    int32_t wave_update;      /* timeadd >= 59/1440 */
    double wave_weight;       /* exp(-33.27 * timeadd') */
    /* shadow ray (device arrays, steps entries) */
    int32_t steps;
    const int32_t* ray_dxdy;  /* [steps][2] (row offset, col offset) */
    const double* ray_dz;     /* [steps] */
    double ray_low, ray_high; int32_t ray_middle;  /* self-shadow azimuth window */
    /* per-patch hour weights (host arrays) */
    float lum[SOLWEIG_MAX_PATCHES];      /* Perez luminance lv_k */
    double yi[SOLWEIG_MAX_PATCHES];      /* min(2 cos(dAzi) tan(alt), 0) */
    uint8_t lw_sun_test[SOLWEIG_MAX_PATCHES]; /* 90 < dAzi < 270 and daytime */
    float band_lsky[SOLWEIG_MAX_BANDS];  /* emissivity * SBC * Tk^4 / pi per band */
    double rad_tot;           /* sum lv * omega * sin(alt) */
    /* UTCI as a polynomial in (Tmrt - Ta), 7 coefficients (scalar weather) */
    double utci[7];
    int32_t utci_valid;       /* 0 -> -999 sentinel */
} SolweigHour;

/* Output planes of one hour; any pointer may be NULL (not written). */
typedef struct SolweigOutputs {
    float* tmrt;
    float* utci;
    float* kdown; float* kup; float* ldown; float* lup;
    float* shadow; float* tg;
    float* keast; float* ksouth; float* kwest; float* knorth;
    float* least; float* lsouth; float* lwest; float* lnorth;
    float* kside_i; float* kside_d; float* kside; float* lside;
    float* d_rad; float* tg_out;
} SolweigOutputs;

/* Thermal state carried from hour to hour (6 planes [pixels], float32). */
typedef struct SolweigState {
    float* tgmap1; float* tgmap1e; float* tgmap1s; float* tgmap1w; float* tgmap1n;
    float* tgout1;
} SolweigState;

const char* solweig_last_error(void);
int solweig_version(void);

/* Walls ------------------------------------------------------------------ */
int solweig_wall_heights(const double* dsm, double* walls, int rows, int cols,
                         double threshold, void* stream);
/* Best template angle (or -1) and template direction (deg; 0 = unresolved)
 * for every wall pixel; the gradient fallback for unresolved pixels is done
 * by the caller on the host.  Templates: line/side1/side2 offset lists
 * (dr, dc) concatenated over 180 angles, with starts[181] per list. */
int solweig_wall_aspect(const double* dsm, const double* walls, double* aspect,
                        int rows, int cols, int radius,
                        const int32_t* line_off, const int32_t* line_start,
                        const int32_t* side1_off, const int32_t* side1_start,
                        const int32_t* side2_off, const int32_t* side2_start,
                        void* stream);

/* Walls from building footprints (src/walls.py:270-332, the geometry wall
 * method).  segments: device float64 [nseg][4] = (u0, v0, u1, v1) in pixel
 * coordinates (the inverse geotransform of the edge's end points; column u,
 * row v), 16-byte aligned.  solweig_wall_segments_burn sets owner[pixels] to
 * the index of the last segment touching each cell (-1: none), where a
 * segment touches every half-open cell [col, col+1) x [row, row+1) holding one
 * of its points (rasterio's all_touched burn with later shapes replacing
 * earlier ones).  solweig_geometry_walls turns owners into float32 planes:
 * walls = the GHSL height where it is >= minimum (float32 compare; NaN/inf
 * read as 0; ghsl may be NULL), else the segment's height; aspect = the
 * segment's aspect mod 360; 0 where no segment touches. */
int solweig_wall_segments_burn(const double* segments, int64_t nseg, int rows, int cols, int32_t* owner,
                               void* stream);
int solweig_geometry_walls(const int32_t* owner, const double* seg_height, const double* seg_aspect,
                           const float* ghsl, int64_t pixels, double minimum, float* walls, float* aspect,
                           void* stream);

/* Shadows ---------------------------------------------------------------- */
/* out: 8 planes [8][pixels] float64 in the reference order
 * (vegsh, sh, vbshvegsh, wallsh, wallsun, wallshve, facesh, facesun);
 * vegetation = 0 runs the building-only variant (planes 1,3,4,6,7 valid). */
int solweig_shadow(const SolweigScene* scene, const int32_t* ray_dxdy, const double* ray_dz,
                   int steps, double low, double high, int middle, int vegetation,
                   double* out, void* stream);

/* Sky view factor -------------------------------------------------------- */
/* Ray tables: per patch p, lengths[p] steps of (dx, dy) and dz in
 * ray_dxdy[p*capacity + n], ray_dz[p*capacity + n].  Writes the packed masks
 * (scene-owned buffer) and planes[16][pixels] float64 in the reference's
 * reduce order (all,E,S,W,N x sh,veg,vb; svftotal). */
int solweig_svf(const double* dsm, const double* vegdem, const double* vegdem2,
                const uint8_t* flags, int rows, int cols,
                int patches, int capacity, const int32_t* ray_dxdy, const double* ray_dz,
                const int32_t* lengths, double hmax,
                const SolweigSkyLayout* layout, const double* band_weights /* [nbands][2] */,
                const uint8_t* sectors /* [patches] bit d: E,S,W,N */,
                double transmissivity, uint32_t* masks, double* planes,
                float* veg_sums, uint8_t* sky_band_counts, void* stream);
/* solweig_svf with the optional packed float4 (dsm, vegdem, vegdem2, 0)
 * geometry of SolweigScene.geo32 (exact float32 values; NULL = the float64
 * rasters): one 16-byte load per ray step, identical masks. */
int solweig_svf_ex(const double* dsm, const double* vegdem, const double* vegdem2,
                   const void* geo32, const uint8_t* flags, int rows, int cols, int patches,
                   int capacity, const int32_t* ray_dxdy, const double* ray_dz,
                   const int32_t* lengths, double hmax, const SolweigSkyLayout* layout,
                   const double* band_weights, const uint8_t* sectors, double transmissivity,
                   uint32_t* masks, double* planes, float* veg_sums, uint8_t* sky_band_counts,
                   void* stream);
/* solweig_svf_ex with a 256-byte aligned device work buffer of
 * solweig_svf_work_bytes(rows, cols) bytes (no counterpart in the reference):
 * per word of 32 patches, upper bounds of the heights ahead along each patch
 * ray let the visibility walks stop early, per-row / per-column exit steps
 * drop their bounds checks, and 16-byte step records (linear offset, dz)
 * replace the offset and dz tables in the walks when capacity <= max(rows,
 * cols) + 2; the masks and planes are identical. */
int64_t solweig_svf_work_bytes(int rows, int cols);
int solweig_svf_ex2(const double* dsm, const double* vegdem, const double* vegdem2,
                    const void* geo32, const uint8_t* flags, int rows, int cols, int patches,
                    int capacity, const int32_t* ray_dxdy, const double* ray_dz,
                    const int32_t* lengths, double hmax, const SolweigSkyLayout* layout,
                    const double* band_weights, const uint8_t* sectors, double transmissivity,
                    uint32_t* masks, double* planes, float* veg_sums, uint8_t* sky_band_counts,
                    void* work, int64_t work_bytes, void* stream);
/* Annulus sums of packed masks (the reduce half of solweig_svf). */
int solweig_svf_reduce(const uint32_t* masks, const double* vegdem2, int64_t pixels,
                       const SolweigSkyLayout* layout, const double* band_weights,
                       const uint8_t* sectors, double transmissivity, double* planes,
                       float* veg_sums, uint8_t* sky_band_counts, void* stream);
/* Pack the reference's float cubes [rows][cols][patches] (shmat, vegshmat,
 * vbshvegshmat) into S/V words (src/model.py:273-284 packs them into bytes). */
int solweig_svf_pack(const float* shmat, const float* vegmat, const float* vbmat, int64_t pixels,
                     int patches, uint32_t* masks, void* stream);
/* Expand packed masks to the reference's float cubes [rows][cols][patches]. */
int solweig_svf_unpack(const uint32_t* masks, int64_t pixels, int patches,
                       float* shmat, float* vegmat, float* vbmat, void* stream);
/* diffsh = shmat - (1 - vegshmat)(1 - transmissivity), float32, any layout. */
int solweig_diffsh(const float* shmat, const float* vegshmat, float* diffsh, int64_t n,
                   float transmissivity, void* stream);

/* Ground view factor ----------------------------------------------------- */
/* Planes [17][pixels] float32 in the reference order. */
int solweig_gvf(const SolweigScene* scene, const float* shadow, const double* wallsun,
                const float* tg, double tgwall, double ta, double ewall, double albedo_b,
                double twater, const int32_t* gvf_dxdy /* [18][steps][2] */, int first_steps,
                int second_steps, float* scratch /* [5][pixels] */, float* planes, void* stream);

/* The hourly step ---------------------------------------------------------- */
/* Hour records and the sky layout live in DEVICE memory (hours[hour]), so a
 * captured launch sequence replays for any forcing.  scratch: [20][pixels]
 * float32: the per-pixel GVF field quad (4), the Lup of the first search
 * direction for water pixels (1) and the 15 GVF planes (15).  Night hours:
 * the shadow and GVF kernels return at once. */
int solweig_step_shadow(const SolweigScene* scene, const SolweigHour* hours, int hour,
                        float* scratch, void* stream);
/* Ground view factors of the hour into scratch (tile_rows: 4, 8 or 16 rows per
 * block).  gvf_dxdy_host: HOST array [18][second_steps][2] of step offsets; it is
 * folded into the kernel parameters (uniform constant-bank reads). */
int solweig_step_gvf(const SolweigScene* scene, const SolweigHour* hours, int hour,
                     const int32_t* gvf_dxdy_host, int first_steps, int second_steps,
                     float* scratch, int tile_rows, void* stream);
int solweig_step_radiation(const SolweigScene* scene, const SolweigSkyLayout* layout,
                           const SolweigHour* hours, int hour, const SolweigState* state,
                           const SolweigOutputs* out, float* scratch, void* stream);
/* All kernels of one hour (gvf_dxdy: host array as for solweig_step_gvf). */
int solweig_step(const SolweigScene* scene, const SolweigSkyLayout* layout,
                 const SolweigHour* hours, int hour, const SolweigState* state,
                 const SolweigOutputs* out, const int32_t* gvf_dxdy, int first_steps,
                 int second_steps, float* scratch, void* stream);
/* All hours of a day: output plane of hour h at base pointer + h * hour_stride. */
int solweig_day(const SolweigScene* scene, const SolweigSkyLayout* layout,
                const SolweigHour* hours, int nhours, const SolweigState* state,
                const SolweigOutputs* base, int64_t hour_stride, const int32_t* gvf_dxdy,
                int first_steps, int second_steps, float* scratch, void* stream);

/* The hourly step with float64 radiation --------------------------------------
 * The reference's precision switch (run.py:27 --dtype float64; src/runtime.py:
 * 43-49 recompiles gvf.cu, shortwave.cu, longwave.cu and flux.cu with Real =
 * double; src/model.py:15-256 then returns float64 planes).  The same hour as
 * solweig_step with every per-pixel radiation quantity in float64: the shadow
 * sh - (1 - vegsh)(1 - psi) unrounded, the Lup excess, the 15 ground view
 * factors, the wave-delay state, the patch sums over every patch in patch
 * order, Kdown/Kup/Kside, Ldown/Lside, Tmrt.  The shadow sweep and the
 * visibility masks are the float32 step's (they are exact).  UTCI stays
 * float32, evaluated from the float32-rounded Tmrt (src/utci.py:8-12).
 * svfbuveg: device float64 [pixels], svf - (1 - svfveg)(1 - transmissivity)
 * of the float32-rounded SVF planes; layout and sky: DEVICE structs; hours64:
 * device array beside hours (same index); scratch: device float64
 * [SOLWEIG_SCRATCH64_PLANES][pixels]. */
#define SOLWEIG_SCRATCH64_PLANES 20
typedef struct SolweigSky64 {
    double omega[SOLWEIG_MAX_PATCHES];          /* steradian */
    double cos_alt[SOLWEIG_MAX_PATCHES];
    double sin_alt[SOLWEIG_MAX_PATCHES];
    double cardinal[4][SOLWEIG_MAX_PATCHES];    /* E,S,W,N longwave direction cosines (0 = off) */
    double diffsh_veg;  /* shmat - (1 - vegshmat)(1 - transmissivity) of a vegetation patch,
                           evaluated in float32 as src/svf.py:117-131 does */
} SolweigSky64;
typedef struct SolweigHour64 {
    double lum[SOLWEIG_MAX_PATCHES];      /* Perez luminance of each patch */
    double band_lsky[SOLWEIG_MAX_BANDS];  /* emissivity * SBC * Tk^4 / pi per band */
} SolweigHour64;
typedef struct SolweigOutputs64 {
    double* tmrt;
    float* utci;
    double* kdown; double* kup; double* ldown; double* lup;
    double* shadow; double* tg;
    double* keast; double* ksouth; double* kwest; double* knorth;
    double* least; double* lsouth; double* lwest; double* lnorth;
    double* kside_i; double* kside_d; double* kside; double* lside;
    double* d_rad; double* tg_out;
} SolweigOutputs64;
typedef struct SolweigState64 {
    double* tgmap1; double* tgmap1e; double* tgmap1s; double* tgmap1w; double* tgmap1n;
    double* tgout1;
} SolweigState64;
int solweig_step64(const SolweigScene* scene, const double* svfbuveg, const SolweigSkyLayout* layout,
                   const SolweigSky64* sky, const SolweigHour* hours, const SolweigHour64* hours64,
                   int hour, const SolweigState64* state, const SolweigOutputs64* out,
                   const int32_t* gvf_dxdy /* host [18][second_steps][2] */, int first_steps,
                   int second_steps, double* scratch, void* stream);

/* Batched day ----------------------------------------------------------------
 * All nhours (<= 64) hours of one day (src/series.py:445-491) in seven
 * launches: shadow sweep and ground view factors for every hour (one launch
 * each), the luminance-weighted sky / vegetation patch sums of all hours as
 * one BF16 tensor-core contraction (tcgen05, FP32 accumulation, weights split
 * into BF16 hi + lo), per-hour sunlit/shaded tables, and one radiation launch
 * whose threads loop over the hours with the wave-delay state in registers.
 * Outputs as solweig_day (plane of hour h at base + h * hour_stride); the
 * cardinal planes (keast..lnorth) must be NULL.  State: tgmap1 and tgout1 are
 * read at the start and written at the end (the four cardinal state planes
 * are not used: their sum is 4 x tgmap1 for any state the model produces).
 * Sky layouts with 145 or 153 patches.  work: device buffer of
 * solweig_day_batched_work_bytes() bytes, 256-byte aligned.  A tensor-core
 * wait that times out sets a device flag read by solweig_day_batched_error. */
int64_t solweig_day_batched_work_bytes(int rows, int cols, int nhours, int has_water);
int solweig_day_batched(const SolweigScene* scene, const SolweigSkyLayout* layout,
                        const SolweigHour* hours, int nhours, const SolweigState* state,
                        const SolweigOutputs* base, int64_t hour_stride, const int32_t* gvf_dxdy,
                        int first_steps, int second_steps, void* work, int64_t work_bytes,
                        void* stream);
/* Launch shapes of the batched day (the autotuner's search space).
 * Defaults (config == NULL): {16, 16, 8, 256, 0, 1, 0, 0}. */
typedef struct SolweigDayConfig {
    int32_t shadow_bx, shadow_by;  /* shadow block: <= 256 threads, a multiple of 32 */
    int32_t gvf_rows;              /* GVF tile rows per block: 4, 8 or 16 (32 columns) */
    int32_t rad_threads;           /* radiation block: 128 or 256 pixels */
    int32_t gemm_ctas_per_sm;      /* contraction CTAs per SM: 0 = as many as fit, 1, 2 */
    int32_t gvf_hours;             /* 1: 32x32 tiles walk all daytime hours in one block, 4
                                      hours per pass (1 m walk, no water); 0: one launch slice
                                      per hour everywhere */
    int32_t no_ceiling;            /* 0: the sweep stops on the per-hour ray ceilings
                                      (same results, fewer steps); 1: every ray walks
                                      to its global clearance */
    int32_t sweep_window;          /* 1 (48x48 px) or 2 (40x40 px): the sweep reads its first
                                      steps from a shared-memory window staged by TMA per 16x16
                                      tile, with the warp-vote exit on the window maximum
                                      (packed float32 geometry, no water; same results);
                                      0: every step from the raster */
} SolweigDayConfig;
int solweig_day_batched_ex(const SolweigScene* scene, const SolweigSkyLayout* layout,
                           const SolweigHour* hours, int nhours, const SolweigState* state,
                           const SolweigOutputs* base, int64_t hour_stride, const int32_t* gvf_dxdy,
                           int first_steps, int second_steps, void* work, int64_t work_bytes,
                           const SolweigDayConfig* config, void* stream);
/* One part of solweig_day_batched_ex (no counterpart in the reference: it
 * lets the host plan later hours while earlier ones run).  part 0: the sweep
 * stage (ray exits, ray ceilings, shadow sweep) of hours [hour_begin,
 * hour_end); the part starting at hour 0 also builds the day's dilated height
 * planes.  part 1: the rest of the day (GVF to radiation) over all hours,
 * hour range ignored.  Part 0 over consecutive ranges covering [0, nhours) in
 * order, then part 1, all on one stream, equals solweig_day_batched_ex. */
int solweig_day_batched_part(const SolweigScene* scene, const SolweigSkyLayout* layout,
                             const SolweigHour* hours, int nhours, const SolweigState* state,
                             const SolweigOutputs* base, int64_t hour_stride, const int32_t* gvf_dxdy,
                             int first_steps, int second_steps, void* work, int64_t work_bytes,
                             const SolweigDayConfig* config, int part, int hour_begin, int hour_end,
                             void* stream);
/* solweig_day_batched_ex timed with CUDA events on `stream` between its
 * stages; synchronises on the last event and writes 5 host floats (ms):
 * shadow, GVF, weights + tables, patch contraction, radiation. */
int solweig_day_batched_timed(const SolweigScene* scene, const SolweigSkyLayout* layout,
                              const SolweigHour* hours, int nhours, const SolweigState* state,
                              const SolweigOutputs* base, int64_t hour_stride,
                              const int32_t* gvf_dxdy, int first_steps, int second_steps,
                              void* work, int64_t work_bytes, const SolweigDayConfig* config,
                              void* stream, float* stage_ms);
/* The scene statics of the batched day's hour-vectorized GVF (no
 * counterpart in the reference): for the 1 m walk (first_steps 1,
 * second_steps 22) of a scene without water, the walk length of every GVF
 * direction (the first building step; device uint32 [4][pixels], 5
 * directions of 6 bits per word) and the albedo-without-shadow GVF (device
 * float32 [pixels]), which depend only on the ground bits and the albedo.
 * Set scene->gvf_hits / gvf_nosh to them and every later day skips that
 * walk; the results are identical. */
int solweig_gvf_statics(const SolweigScene* scene, const int32_t* gvf_dxdy, int first_steps, int second_steps,
                        uint32_t* hits, float* nosh, void* stream);
/* Byte offsets inside the batched-day work buffer: quads [H][px] float4,
 * first-direction Lup [H][px], GVF [H][3][px] (Lup, albedo, shadow),
 * albedo-without-shadow GVF [px], patch sums (room for [2][2H][px]; the day
 * writes [2H][px]: sky plus 0.03 x vegetation sums of luminance and
 * luminance*cos*omega per hour), weights f32 [2H][160], BF16 operands (hi/lo
 * of the weights and of 0.03 x the weights), per-hour tables, error flag pair
 * (placed first, at offset 0 for every raster size), 16x16 tile maxima of the
 * heights (window sweep), total size: offsets[0..10]. */
int solweig_day_batched_layout(int rows, int cols, int nhours, int has_water, int64_t* offsets);
/* Copy the device error flag of the last batched day in `work` to out_device:
 * 0 = none, 1 = a tensor-core wait of the contraction timed out (results
 * invalid), 2 = a sweep window's TMA wait timed out (that tile walked from the
 * raster instead; results still exact), 3 = a sun ray table stayed inside the
 * raster for more than max(rows, cols) + 2 steps (that hour's results
 * invalid; rays built as the reference builds them never do).  The int after
 * the flag in `work` has bit v set for every flag v raised by any day run in
 * that buffer since the caller last zeroed it (the days never clear it), so
 * one read after a graph of many days or tiles covers all of them. */
int solweig_day_batched_error(const void* work, int rows, int cols, int nhours, int has_water,
                              int* out_device, void* stream);
/* The patch contraction alone: out[c][p] = sum_k sky(p,k) * weights[c][k] for
 * c < ncols and out[ncols + c][p] = sum_k veg(p,k) * weights[c][k], with
 * sky = S & ~V and veg = S & V of the packed masks; weights: device float32
 * [ncols][160] (ncols <= 256), contracted as BF16 hi + lo with FP32
 * accumulation.  work: >= 4 * 16*ceil(ncols/16) * 160 + 16 bytes, 16-byte aligned. */
int solweig_patch_sums(const uint32_t* masks, int64_t pixels, int patches, const float* weights,
                       int ncols, float* out, void* work, int64_t work_bytes, void* stream);

/* Day gradient ---------------------------------------------------------------
 * Reverse pass of the batched day with the shadow and SVF masks held fixed
 * (the 1 m GVF walk, first = 1, second = 22; no water pixels; nhours <= 32).
 * Per-pixel parameters replace the scene's ground albedo and emissivity and
 * the hour's psi (direct-beam transmissivity of vegetation in
 * shadow = sh - (1 - vegsh)(1 - t)).  objective: 0 = daily mean UTCI (NaN on
 * roofs), 1 = daily mean Tmrt.  Both entry points recompute the day from its
 * inputs (nothing is kept between calls).  The backward pass returns dJ/d
 * parameter for J = sum_p weights[p] * daily[p], and the partials of J with
 * respect to the hour scalars the device consumes:
 * hour_grad[h][SOLWEIG_GRAD_HOUR_FIELDS] = (ta, rad_i, rad_d, rad_tot, ci_tgg,
 * tgwall, band_lsky[8], utci[7]) and lum_grad[h][4][160] = mask-transposed
 * sums (sky, sky x cos*omega, vegetation, vegetation x cos*omega) of the
 * adjoints of the contraction outputs, from which
 * dJ/dlum_k = lum_grad[h][0][k] + lum_grad[h][2][k]
 *           + cos_alt_k * omega_k * (lum_grad[h][1][k] + lum_grad[h][3][k]). */
#define SOLWEIG_GRAD_HOUR_FIELDS 21
typedef struct SolweigGradParams {
    const float* albedo;          /* [pixels] */
    const float* emissivity;      /* [pixels] */
    const float* transmissivity;  /* [pixels] */
} SolweigGradParams;
int64_t solweig_day_grad_work_bytes(int rows, int cols, int nhours);
int solweig_day_grad_forward(const SolweigScene* scene, const SolweigSkyLayout* layout,
                             const SolweigHour* hours, int nhours, const int32_t* gvf_dxdy,
                             int first_steps, int second_steps, const SolweigGradParams* params,
                             int objective, double* daily /* [pixels] */, void* work,
                             int64_t work_bytes, void* stream);
int solweig_day_grad_backward(const SolweigScene* scene, const SolweigSkyLayout* layout,
                              const SolweigHour* hours, int nhours, const int32_t* gvf_dxdy,
                              int first_steps, int second_steps, const SolweigGradParams* params,
                              int objective, const float* weights, float* d_albedo,
                              float* d_emissivity, float* d_transmissivity, double* hour_grad,
                              double* lum_grad, void* work, int64_t work_bytes, void* stream);

/* solweig_step without a scratch argument -- no counterpart in the reference.
 * For callers that cannot allocate device memory: a host model that owns its
 * arrays but no device allocator for temporaries, or that must not call
 * cudaMalloc/cudaFree inside its time loop (cudaFree synchronises the device).
 * The [20][pixels] scratch lives in a file-scope static device array of
 * SOLWEIG_STEP_SCRATCH_PLANES x SOLWEIG_STATIC_SCRATCH_MAX_PIXELS floats
 * (20 MiB); tiles above SOLWEIG_STATIC_SCRATCH_MAX_PIXELS pixels are rejected
 * with SOLWEIG_ERR_INVALID.  Nothing is allocated.  The first call on each
 * device (with that device current) looks the array's address up once; make
 * that first call before any stream capture.  The array is shared by every
 * call on a device: two calls that overlap in time (different streams or
 * host threads) race on it and must be serialised by the caller.  Nothing in
 * the array has to start at zero. */
#define SOLWEIG_STEP_SCRATCH_PLANES 20
#define SOLWEIG_STATIC_SCRATCH_MAX_PIXELS (512 * 512)
int solweig_step_static_scratch(const SolweigScene* scene, const SolweigSkyLayout* layout,
                                const SolweigHour* hours, int hour, const SolweigState* state,
                                const SolweigOutputs* out, const int32_t* gvf_dxdy,
                                int first_steps, int second_steps, void* stream);

/* Static scene preparation (src/series.py:252-349) ------------------------- */
/* classes: [nclasses][6] (code, albedo, emissivity, TgK, Tstart, TmaxLST);
 * defaults: albedo, emissivity, TgK, Tstart, TmaxLST without land cover;
 * landcover_in may be NULL. */
int solweig_scene_build(const double* dsm_in, const double* trees_in, const double* dem_in,
                        const double* landcover_in, int64_t pixels, double raise_dsm,
                        double raise_dem, const double* classes, int nclasses,
                        const double* defaults, double* dsm, double* vegdem, double* vegdem2,
                        uint8_t* flags, float* alb, float* emis, float* tgk, float* tstart,
                        float* tmaxlst, float* lc_out, void* stream);
/* From the 16 SVF planes: float32 copies of the 15 SVF planes, svfbuveg,
 * svfalfa, tan(asvf) and the 18 GVF wall-face bits (face windows from the host). */
int solweig_scene_finalize(const double* planes, const double* walls, const double* aspect_rad,
                           int64_t pixels, double transmissivity, const double* face_low,
                           const double* face_high, const int32_t* face_middle, float* svf32,
                           float* svfbuveg, double* svfalfa, double* tan_asvf, uint32_t* gvf_face,
                           void* stream);

/* UTCI ------------------------------------------------------------------- */
/* Per-pixel weather (any of ta/rh/va may be a 1-element array when its
 * *_scalar flag is set). */
int solweig_utci(const float* ta, const float* rh, const float* tmrt, const float* va,
                 int ta_scalar, int rh_scalar, int va_scalar, float* out, int64_t n,
                 void* stream);
/* Scalar weather for the whole raster (src/kernels/utci.cu:243-523): the
 * polynomial is collapsed on the host and evaluated per pixel in (Tmrt - Ta). */
int solweig_utci_scalar(double ta, double rh, double va, const float* tmrt, float* out, int64_t n,
                        void* stream);
/* Host function: UTCI as a polynomial in D = Tmrt - Ta for scalar weather,
 * coefficients[0..6] (all zero when an input is the -999 sentinel). */
int solweig_utci_collapse(double ta, double rh, double va, double* coefficients);

/* sizeof(SolweigScene, SolweigSkyLayout, SolweigHour, SolweigOutputs, SolweigState). */
int solweig_struct_sizes(int64_t* out);
/* sizeof(SolweigSky64, SolweigHour64, SolweigOutputs64, SolweigState64). */
int solweig_struct_sizes64(int64_t* out);

#ifdef __cplusplus
}
#endif
#endif /* SOLWEIG_B200_H */
