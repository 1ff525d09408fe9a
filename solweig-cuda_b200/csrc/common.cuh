// Shared device/host helpers of libsolweig_b200 (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#include "../../include/solweig_b200.h"

namespace solweig {

// Thread-local last-error message, set by every failing entry point.
void set_error(const char* fmt, ...);

#define SOLWEIG_CHECK_ARG(cond, ...)                 \
    do {                                             \
        if (!(cond)) {                               \
            ::solweig::set_error(__VA_ARGS__);       \
            return SOLWEIG_ERR_INVALID;              \
        }                                            \
    } while (0)

#define SOLWEIG_CHECK_LAUNCH(what)                                                      \
    do {                                                                                \
        cudaError_t _e = cudaGetLastError();                                            \
        if (_e != cudaSuccess) {                                                        \
            ::solweig::set_error("%s: %s", what, cudaGetErrorString(_e));               \
            return SOLWEIG_ERR_CUDA;                                                    \
        }                                                                               \
    } while (0)

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

constexpr double kSBC = 5.67051e-8;
constexpr double kPi = 3.141592653589793238462643383279502884;

// Number of blocks for a 1-D launch over n items.
inline unsigned blocks_for(long long n, int threads) {
    return static_cast<unsigned>((n + threads - 1) / threads);
}

// Steps covered by the window maximum of the ray-ceiling planes (ceiling.cuh):
// a walk may skip that many steps at once on it (shadow.cuh).
constexpr int kCeilSkip = 8;

__device__ __forceinline__ bool in_raster(int r, int c, int rows, int cols) {
    return (unsigned)r < (unsigned)rows && (unsigned)c < (unsigned)cols;
}

__host__ __device__ __forceinline__ double pow4(double x) {
    double x2 = x * x;
    return x2 * x2;
}

// Error flag pair of a batched day's work buffer: word 0 = the last flag of
// the current day (cleared when the day starts), word 1 = bit v set for every
// flag v raised since the host last zeroed it (never cleared by the kernels).
__device__ __forceinline__ void raise_day_flag(int* error, int value) {
    atomicExch(error, value);
    atomicOr(error + 1, 1 << value);
}

}  // namespace solweig
