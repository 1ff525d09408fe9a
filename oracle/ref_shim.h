/* Host shim that lets the reference's CUDA C kernel files compile as plain
 * C++ for the CPU, unchanged and in place (test infrastructure only).
 *
 * The kernels index work with blockIdx/blockDim/threadIdx; ref_driver.cpp sets
 * these globals and calls each kernel body once per (block, thread).  The
 * round-to-nearest intrinsics map to the plain IEEE operators; the driver is
 * compiled with -ffp-contract=off so no FMA contraction changes a rounding.
 */
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>

struct RefDim3 { unsigned x, y, z; };
extern RefDim3 blockIdx, blockDim, threadIdx, gridDim;

#define __global__
#define __device__
#define __host__
#define __forceinline__ inline
#define __align__(n) alignas(n)
#define __restrict__

static inline float __fsub_rn(float a, float b) { return a - b; }
static inline float __fadd_rn(float a, float b) { return a + b; }
static inline float __fmul_rn(float a, float b) { return a * b; }
static inline float __fdiv_rn(float a, float b) { return a / b; }
static inline double __dsub_rn(double a, double b) { return a - b; }
static inline double __dadd_rn(double a, double b) { return a + b; }
static inline double __dmul_rn(double a, double b) { return a * b; }
static inline double __ddiv_rn(double a, double b) { return a / b; }
