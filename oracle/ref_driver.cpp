/* CPU driver around the reference's own kernel sources (test infrastructure).
 *
 * Built by oracle/Makefile, which passes -DREF_KERNELS=<reference>/src/kernels
 * so that the reference files are compiled from where they lie; nothing of
 * the reference is copied into this repository.  Each ref_* entry point runs
 * the named reference kernel over its whole launch grid on one CPU thread.
 *
 *   ref_utci_scalar      utci.cu:243-523  (scalar-weather prepare + integrate)
 *   ref_utci_fused       utci.cu:1-241    (per-pixel weather)
 *   ref_wall_heights     geometry.cu:15-34
 *   ref_wall_directions  geometry.cu:36-63
 *   ref_svf_visibility   geometry.cu:77-119
 *   ref_svf_reduce       geometry.cu:121-159
 *   ref_shadow_pixels    geometry.cu:185-253
 */
#include "ref_shim.h"

RefDim3 blockIdx, blockDim, threadIdx, gridDim;

#define REF_STR2(x) #x
#define REF_STR(x) REF_STR2(x)
#include REF_STR(REF_KERNELS/utci.cu)
#include REF_STR(REF_KERNELS/geometry.cu)

static void set_linear(unsigned block, unsigned y = 0) {
    blockIdx = {block, y, 0};
    blockDim = {1, 1, 1};
    threadIdx = {0, 0, 0};
    gridDim = {1, 1, 1};
}

extern "C" {

int ref_utci_scalar(float ta, float rh, float va, const float* tmrt, float* out,
                    long long n, double* coefficients) {
    set_linear(0);
    for (int i = 0; i < 7; ++i) coefficients[i] = 0.0;
    utci_scalar_weather_prepare(&ta, &rh, &va, coefficients);
    utci_scalar_weather_integrate(&ta, &rh, tmrt, &va, coefficients, out, n);
    return 0;
}

int ref_utci_fused(const float* ta, const float* rh, const float* tmrt, const float* va,
                   float* out, long long n) {
    set_linear(0);
    utci_fused_kernel(ta, rh, tmrt, va, out, n);
    return 0;
}

int ref_wall_heights(const double* dsm, double* walls, int rows, int cols, double threshold) {
    long long n = (long long)rows * cols;
    for (long long p = 0; p < n; ++p) {
        set_linear((unsigned)p);
        wall_heights(dsm, walls, rows, cols, threshold);
    }
    return 0;
}

int ref_wall_directions(const unsigned char* walls, const long long* pixels, long long count,
                        const long long* offsets, const int* starts, int rows, int cols,
                        int radius, short* angles) {
    for (long long i = 0; i < count; ++i) {
        set_linear((unsigned)i);
        wall_directions(walls, pixels, count, offsets, starts, rows, cols, radius, angles);
    }
    return 0;
}

int ref_svf_visibility(const float* a, const float* top, const float* bottom,
                       const double* a64, const double* top64, const double* bottom64,
                       const unsigned char* bushplant, int rows, int cols, int patches,
                       int capacity, const int* offsets, const float* heights,
                       const double* heights64, const int* lengths,
                       float* shmat, float* vegmat, float* vbmat) {
    long long n = (long long)rows * cols;
    for (int patch = 0; patch < patches; ++patch)
        for (long long p = 0; p < n; ++p) {
            set_linear((unsigned)p, (unsigned)patch);
            svf_visibility(a, top, bottom, a64, top64, bottom64, bushplant, rows, cols,
                           patches, capacity, offsets, heights, heights64, lengths, 0,
                           patches, shmat, vegmat, vbmat);
        }
    return 0;
}

int ref_svf_reduce(const float* shmat, const float* vegmat, const float* vbmat,
                   const double* bottom, const unsigned char* sectors, const int* band_offsets,
                   const double* weights, long long pixels, int patches, int bands,
                   double trans, double* output) {
    for (long long p = 0; p < pixels; ++p) {
        set_linear((unsigned)p);
        svf_reduce(shmat, vegmat, vbmat, bottom, sectors, band_offsets, weights, pixels,
                   patches, bands, trans, output);
    }
    return 0;
}

int ref_shadow_pixels(const double* fields, const float* scan, const int* offsets,
                      const double* heights, const float* fast_heights, int steps,
                      int rows, int cols, double low, double high, int middle, int vegetation,
                      double* out) {
    long long n = (long long)rows * cols;
    for (long long p = 0; p < n; ++p) {
        set_linear((unsigned)p);
        shadow_pixels(fields, scan, offsets, heights, fast_heights, steps, rows, cols, low,
                      high, middle, vegetation, out);
    }
    return 0;
}

}  // extern "C"
