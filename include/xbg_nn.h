/*
 * xbg_nn.h -- C ABI of the wave surrogate's device kernels (libxbg_b200.so).
 *
 * No counterpart in the reference: the surrogate is a convolutional network
 * that stands in for the wave action sub-steps between flow updates.  Its
 * arithmetic runs on hand-written sm_100a kernels: a tensor-core GEMM
 * (tcgen05, bf16 operands, fp32 accumulators in tensor memory) and the
 * convolution / pooling / optimiser kernels around it.  All pointers are
 * device pointers; calls enqueue on `stream` and do not synchronise.
 */
#ifndef XBG_NN_H
#define XBG_NN_H
#include <stddef.h>
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

#define XBG_NN_RELU      1   /* epilogue: max(x, 0)            */
#define XBG_NN_OUT_BF16  2   /* epilogue: store bf16 (else f32) */
#define XBG_NN_ATOMIC    4   /* epilogue: atomically add into f32 C (split-K
                                partials; no bias or activation)          */

/* C[M x N] = act(A[M x K] . B[N x K]^T + bias[N]); A, B bf16 row-major (K
 * contiguous, leading dimensions lda/ldb in elements, multiples of 8, 16-B
 * aligned), C f32 or bf16 row-major (ldc); bias f32 or NULL.  N in 16..256
 * (one of 16, 32, 48, 64, 96, 128, 192, 256), K a multiple of 64.  *err (a
 * device int the caller zeroes) receives XBG_ERR_TIMEOUT if a bounded
 * tensor-core wait ran out.                                                 */
int xbg_nn_gemm(const void* A, const void* B, const float* bias, void* C,
                int M, int N, int K, int lda, int ldb, int ldc, int flags,
                int ksplit, int* err, void* stream);
/* ksplit > 1 (requires XBG_NN_ATOMIC): the K chunks are split over ksplit
 * CTAs per row tile, each adding its partial product into C.              */

#ifdef __cplusplus
}
#endif
#endif /* XBG_NN_H */
