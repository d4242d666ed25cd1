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
#define XBG_NN_CHECK_TIMEOUT 8  /* xbg_nn_gemm only: check of the time-out
                                exit.  Every CTA waits, with a short limit,
                                on a barrier that nothing completes, then
                                leaves as a stalled pipeline does: no MMA
                                issued, C untouched, tensor memory freed,
                                *err = XBG_ERR_TIMEOUT.                    */

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

/* 3x3 convolution with zero padding as an implicit GEMM on the tensor cores:
 * Y[p][n] = act(sum over tap, c of X[b, y+dy, x+dx, c] Wt[n][tap*cin + c]
 * + bias[n]) for the B*H*W pixels p of the NHWC bf16 input X (channel
 * stride ldx), n < N (16..256, a multiple of 16), tap = (dy+1)*3 + dx+1; the
 * weights' columns 9*cin..Kp-1 are ignored (Kp a multiple of 64).  Same
 * result as xbg_nn_im2col3x3 followed by xbg_nn_gemm, without the im2col
 * matrix.  flags: XBG_NN_RELU, XBG_NN_OUT_BF16 (else fp32 Y).             */
int xbg_nn_conv3x3(const void* X, const void* Wt, const float* bias, void* Y,
                   int B, int H, int W, int cin, int ldx, int N, int Kp,
                   int ldw, int ldy, int flags, int* err, void* stream);

/* Input movement of xbg_nn_conv3x3 where the shape tiles (128-pixel tiles of
 * whole rows or of 128-pixel row pieces, channel counts a multiple of 16):
 * on (1, the default) the tensor memory accelerator copies each tap's input
 * box into shared memory; off (0) every thread gathers 16-byte pieces.  The
 * results are identical; the switch exists for comparison.                */
int xbg_nn_conv_set_tma(int on);
/* Weight and bias gradient of xbg_nn_conv3x3 as an implicit GEMM over the
 * pixels: gw[n][tap*cin + c] (+)= sum over p of dz[p][n] X[b, y+dy, x+dx, c]
 * and, when gb is not NULL, gb[n] (+)= sum over p of dz[p][n], for n < N
 * (16, 32, 48, 64, 96, 128, 192 or 256; dz bf16 [P][ldz], ldz >= N); adds
 * when accumulate, else stores (columns 9*cin.. of gw untouched).  The
 * pixels are split into ksplit ranges whose partial sums go to `work` (at
 * least xbg_nn_conv3x3_wgrad_work(cin, N, ksplit) floats, 16-B aligned) and
 * are added in a fixed order: the result does not depend on scheduling.
 * X: the convolution's NHWC bf16 input (B*H*W pixels, channel stride ldx,
 * cin a multiple of 8, 16-B aligned); gw f32 [N][ldw], ldw >= 9*cin; *err
 * receives XBG_ERR_TIMEOUT if a bounded tensor-core wait ran out.          */
long long xbg_nn_conv3x3_wgrad_work(int cin, int N, int ksplit);
int xbg_nn_conv3x3_wgrad(const void* X, const void* Dz, float* gw, float* gb,
                         float* work, int B, int H, int W, int cin, int ldx,
                         int N, int ldz, int ldw, int ksplit,
                         int accumulate, int* err, void* stream);

/* Weights of the input-gradient convolution: wf[c][tap*cd + n] =
 * w[n][(8-tap)*cin + c] for c < cin, n < cd (w has at least cd rows, zero
 * beyond the layer's outputs), columns 9*cd..ldf-1 zero.  With them
 * xbg_nn_conv3x3 of dz (cd channels) gives dx = the gradient of the
 * convolution's input.                                                      */
int xbg_nn_conv3x3_flip(const void* w, int ldw, int cin, int cd, void* wf,
                        int ldf, void* stream);

/* Training crops: dst[b] = the crop x crop window of image idx[3b] of src
 * ([images][ny][nx] pixels of bytes_per_px bytes, a multiple of 4) whose
 * first row and column are idx[3b+1], idx[3b+2] (a DEVICE int array; the
 * caller keeps the windows inside the images).                             */
int xbg_nn_gather_crops(const void* src, void* dst, const int* idx, int B,
                        int ny, int nx, int crop, int bytes_per_px,
                        void* stream);

/* ---- layers around the GEMM (NHWC bf16 tensors, [pixels][channels], the
 * channel counts multiples of 8) ------------------------------------------ */
/* col[p][tap*C + c] = x[b, y+dy, x+dx, c] (0 outside the image; tap = (dy+1)*3
 * + dx+1); columns 9C..Kp-1 and rows B*H*W..Mpad-1 are zero.  Kp % 64 == 0. */
int xbg_nn_im2col3x3(const void* x, void* col, int B, int H, int W, int C,
                     int Kp, int Mpad, void* stream);
/* dx (+)= the gather of dcol back onto the pixels it was taken from. */
int xbg_nn_col2im3x3(const void* dcol, void* dx, int B, int H, int W, int C,
                     int Kp, int accumulate, void* stream);
/* dst[c][r] = src[r][c], r < R, c < Cc (bf16). */
int xbg_nn_transpose(const void* src, void* dst, int R, int Cc, int lds,
                     int ldd, void* stream);
/* dx = dy where y > 0 (n values, a multiple of 8). */
int xbg_nn_relu_bwd(const void* dy, const void* y, void* dx, long long n,
                    void* stream);
/* db[n] += sum over p < P of dy[p][n] (f32 db, N <= 256). */
int xbg_nn_bias_grad(const void* dy, float* db, int P, int N, int ld,
                     void* stream);
/* 2x2 average pooling and its backward (dx (+)= dy / 4 on each child). */
int xbg_nn_pool2(const void* x, void* y, int B, int H, int W, int C,
                 void* stream);
int xbg_nn_pool2_bwd(const void* dy, void* dx, int B, int H, int W, int C,
                     int accumulate, void* stream);
/* nearest 2x upsampling of x[B,h,w,C] into channels [c0, c0+C) of
 * y[B,2h,2w,ldy], and its backward (sum of the four children). */
int xbg_nn_up2(const void* x, void* y, int B, int h, int w, int C, int ldy,
               int c0, void* stream);
int xbg_nn_up2_bwd(const void* dy, void* dx, int B, int h, int w, int C,
                   int ldy, int c0, void* stream);
/* x[P][C] -> channels [c0, c0+C) of y[P][ldy] (concatenation), or back
 * (reverse = 1, optionally adding into x). */
int xbg_nn_chan_copy(void* x, void* y, long long P, int C, int ldy, int c0,
                     int reverse, int accumulate, void* stream);
/* mean squared error of pred[P][ldp] (f32) against tgt[P][nc] (f32):
 * *loss += mean, dpred[P][ldg] (bf16, ldg a multiple of 8, 16-B aligned) =
 * its gradient (0 in padding). */
int xbg_nn_mse(const float* pred, const float* tgt, void* dpred, float* loss,
               int P, int nc, int ldp, int ldg, void* stream);
/* Adam step `step` (1-based) on f32 master weights p with bf16 copy pb. */
int xbg_nn_adam(float* p, void* pb, const float* g, float* m, float* v,
                long long n, float lr, float b1, float b2, float eps, int step,
                void* stream);
int xbg_nn_to_bf16(const float* a, void* b, long long n, void* stream);
/* dst[c][p] = src[c][p] for nc planes (DEVICE arrays of plane pointers). */
int xbg_nn_copy_planes(const float* const* src, float* const* dst, int nc,
                       long long P, void* stream);
/* network input from model planes: x[p][c] = bf16((planes[c][p] - mean[c])
 * * inv_std[c]); planes is a DEVICE array of nc f32 plane pointers (NULL =
 * a zero plane).                                                           */
int xbg_nn_encode(const float* const* planes, int nc, const float* mean,
                  const float* inv_std, void* x, long long P, void* stream);
/* xbg_nn_encode for nimg images of different sizes padded to one Hp x Wp
 * batch ([nimg][Hp][Wp][nc] bf16): image b has dims[2b] x dims[2b+1]
 * (<= Wp x Hp) pixels and planes planes[b*nc + c]; a NULL plane is the
 * constant cval[b*nc + c] (or 0 when cval is NULL); pixels beyond the image
 * repeat its last column and row.  planes, dims, cval: DEVICE arrays.      */
int xbg_nn_encode_batch(const float* const* planes, int nc, const int* dims,
                        const float* cval, const float* mean,
                        const float* inv_std, void* x, int nimg, int Hp,
                        int Wp, void* stream);
/* xbg_nn_decode for such a batch: out [nimg][Hp][Wp][ldo] f32; hold, dst
 * and (optional, may be NULL) dst0 are DEVICE arrays of nimg*nc plane
 * pointers; dst0 receives a copy of hold.  Only each image's own pixels
 * are written.                                                             */
int xbg_nn_decode_batch(const float* out, int ldo, const float* const* hold,
                        const float* ym, const float* ys, float* const* dst,
                        float* const* dst0, const int* dims, int nc, int nimg,
                        int Hp, int Wp, void* stream);
/* network output to model planes: dst[c][p] = hold[c][p] + out[p][c] *
 * ys[c] + ym[c]; hold and dst are DEVICE arrays of nc f32 plane pointers. */
int xbg_nn_decode(const float* out, int ldo, const float* const* hold,
                  const float* ym, const float* ys, float* const* dst, int nc,
                  long long P, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* XBG_NN_H */
