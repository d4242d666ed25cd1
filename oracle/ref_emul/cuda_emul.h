/*
 * cuda_emul.h -- TEST INFRASTRUCTURE ONLY.
 *
 * Just enough of the CUDA C++ dialect for the reference's kernel files
 * (Wave_kernel.cu, Flow_kernel.cu, Sediment_kernel.cu) to compile as host C++
 * and run on the CPU with a serial launch loop.  The reference files are
 * compiled in place from the reference checkout; nothing of them is copied.
 *
 * Semantics: one emulated thread per block (blockDim = 1x1x1), blocks run in
 * order iy-outer / ix-inner.  The reference kernels use __shared__ arrays only
 * as per-thread slots [tx][ty], so a serial run of the threads is exact.
 * min/max on floats follow CUDA's fminf/fmaxf; mixed float/double arguments
 * promote to double as CUDA's math overloads do.
 */
#ifndef XBG_CUDA_EMUL_H
#define XBG_CUDA_EMUL_H
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

struct dim3 { unsigned x, y, z; };
extern dim3 threadIdx, blockIdx, blockDim, gridDim;

#define __global__
#define __device__
#define __host__
#define __forceinline__ inline
#define __shared__ static
static inline void __syncthreads() {}

static inline float min(float a, float b) { return fminf(a, b); }
static inline float max(float a, float b) { return fmaxf(a, b); }
static inline double min(double a, double b) { return fmin(a, b); }
static inline double max(double a, double b) { return fmax(a, b); }
static inline double min(float a, double b) { return fmin((double)a, b); }
static inline double max(float a, double b) { return fmax((double)a, b); }
static inline double min(double a, float b) { return fmin(a, (double)b); }
static inline double max(double a, float b) { return fmax(a, (double)b); }
static inline int min(int a, int b) { return a < b ? a : b; }
static inline int max(int a, int b) { return a > b ? a : b; }
static inline unsigned min(unsigned a, unsigned b) { return a < b ? a : b; }
static inline unsigned max(unsigned a, unsigned b) { return a > b ? a : b; }

#endif
