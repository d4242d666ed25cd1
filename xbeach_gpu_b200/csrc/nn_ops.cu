// nn_ops.cu -- the wave surrogate's kernels around the tensor-core GEMM.
//
// Activations are NHWC bf16 tensors stored as [pixels][channels] (channel
// counts multiples of 8, so every access moves 16 B).  A 3x3 convolution is
//   im2col:  col[p][tap*C + c] = x[b, y+dy, x+dx, c] (zero outside), K padded
//            to a multiple of 64 with zeros,
//   GEMM:    y[p][n] = act(col[p] . W[n] + bias[n])            (nn_gemm.cu)
// and its backward is
//   dcol = dy . W (GEMM on W^T), dx = col2im(dcol) (a gather over the nine
//   taps, no atomics), dW += dy^T . col (GEMM on the transposes, split-K),
//   dbias = column sums of dy.
// The U-Net around it: 2x2 average pooling, nearest 2x upsampling, channel
// concatenation, and their backwards; the loss (mean squared error of the
// normalised outputs) and the Adam update of fp32 master weights with their
// bf16 copies.
#include <cuda_bf16.h>
#include <cstdint>

#include "../../include/xbg.h"
#include "../../include/xbg_nn.h"

namespace xbg {
namespace nn {

typedef __nv_bfloat16 bf;

__device__ __forceinline__ void unpack8(const uint4& v, float* f) {
    const __nv_bfloat162* h = reinterpret_cast<const __nv_bfloat162*>(&v);
#pragma unroll
    for (int k = 0; k < 4; k++) {
        float2 t = __bfloat1622float2(h[k]);
        f[2 * k] = t.x;
        f[2 * k + 1] = t.y;
    }
}
__device__ __forceinline__ uint4 pack8(const float* f) {
    uint4 v;
    __nv_bfloat162* h = reinterpret_cast<__nv_bfloat162*>(&v);
#pragma unroll
    for (int k = 0; k < 4; k++) h[k] = __floats2bfloat162_rn(f[2 * k], f[2 * k + 1]);
    return v;
}

constexpr int TPB = 256;
inline unsigned blocks_for(long long n) { return (unsigned)((n + TPB - 1) / TPB); }

// one thread per (pixel p < Mpad, 8-wide group of K)
__global__ void k_im2col(const bf* __restrict__ x, bf* __restrict__ col, int B, int H, int W, int C, int Kp, int Mpad) {
    const long long G = Kp / 8;
    long long idx = (long long)blockIdx.x * TPB + threadIdx.x;
    if (idx >= (long long)Mpad * G) return;
    const int p = (int)(idx / G), k = (int)(idx % G) * 8;
    uint4 v = make_uint4(0, 0, 0, 0);
    if (p < B * H * W && k < 9 * C) {
        const int tap = k / C, c = k - tap * C;
        const int b = p / (H * W), r = p - b * H * W, y = r / W, xx = r - y * W;
        const int ys = y + tap / 3 - 1, xs = xx + tap % 3 - 1;
        if (ys >= 0 && ys < H && xs >= 0 && xs < W) v = *(const uint4*)(x + ((size_t)(b * H + ys) * W + xs) * C + c);
    }
    *(uint4*)(col + (size_t)p * Kp + k) = v;
}

// dx[b,y,x,c] (+)= sum over taps of dcol[(b, y-dy, x-dx)][tap*C + c]
__global__ void k_col2im(const bf* __restrict__ dcol, bf* __restrict__ dx, int B, int H, int W, int C, int Kp,
                         int accumulate) {
    const int G = C / 8;
    long long idx = (long long)blockIdx.x * TPB + threadIdx.x;
    if (idx >= (long long)B * H * W * G) return;
    const int p = (int)(idx / G), c = (int)(idx % G) * 8;
    const int b = p / (H * W), r = p - b * H * W, y = r / W, xx = r - y * W;
    float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
    for (int tap = 0; tap < 9; tap++) {
        const int yq = y - (tap / 3 - 1), xq = xx - (tap % 3 - 1);
        if (yq < 0 || yq >= H || xq < 0 || xq >= W) continue;
        float f[8];
        unpack8(*(const uint4*)(dcol + (size_t)((b * H + yq) * W + xq) * Kp + tap * C + c), f);
#pragma unroll
        for (int j = 0; j < 8; j++) acc[j] += f[j];
    }
    uint4* o = (uint4*)(dx + (size_t)p * C + c);
    if (accumulate) {
        float f[8];
        unpack8(*o, f);
#pragma unroll
        for (int j = 0; j < 8; j++) acc[j] += f[j];
    }
    *o = pack8(acc);
}

// dst[c][r] = src[r][c] for r < R, c < Cc (32 x 32 tiles through shared memory)
__global__ void k_transpose(const bf* __restrict__ src, bf* __restrict__ dst, int R, int Cc, int lds, int ldd) {
    __shared__ bf t[32][33];
    const int r0 = blockIdx.x * 32, c0 = blockIdx.y * 32;
    for (int k = threadIdx.y; k < 32; k += 8) {
        int r = r0 + k, c = c0 + threadIdx.x;
        t[k][threadIdx.x] = (r < R && c < Cc) ? src[(size_t)r * lds + c] : __float2bfloat16(0.0f);
    }
    __syncthreads();
    for (int k = threadIdx.y; k < 32; k += 8) {
        int c = c0 + k, r = r0 + threadIdx.x;
        if (c < Cc && r < R) dst[(size_t)c * ldd + r] = t[threadIdx.x][k];
    }
}

// dx = dy where y > 0 (ReLU backward), 8 per thread
__global__ void k_relu_bwd(const bf* __restrict__ dy, const bf* __restrict__ y, bf* __restrict__ dx, long long n8) {
    long long i = (long long)blockIdx.x * TPB + threadIdx.x;
    if (i >= n8) return;
    float a[8], b[8];
    unpack8(((const uint4*)dy)[i], a);
    unpack8(((const uint4*)y)[i], b);
#pragma unroll
    for (int j = 0; j < 8; j++) a[j] = b[j] > 0.0f ? a[j] : 0.0f;
    ((uint4*)dx)[i] = pack8(a);
}

// db[n] += sum over p < P of dy[p][n] (n < N); one block per 256 pixels
__global__ void k_bias_grad(const bf* __restrict__ dy, float* __restrict__ db, int P, int N, int ld) {
    __shared__ float s[256];
    for (int n = threadIdx.x; n < N; n += TPB) s[n] = 0.0f;
    __syncthreads();
    const int p0 = blockIdx.x * 256;
    for (int e = threadIdx.x; e < 256 * N; e += TPB) {
        int p = p0 + e / N, n = e % N;
        if (p < P) atomicAdd(&s[n], __bfloat162float(dy[(size_t)p * ld + n]));
    }
    __syncthreads();
    for (int n = threadIdx.x; n < N; n += TPB) atomicAdd(&db[n], s[n]);
}

// 2x2 average pooling of x[B, H, W, C] -> y[B, H/2, W/2, C]
__global__ void k_pool2(const bf* __restrict__ x, bf* __restrict__ y, int B, int H, int W, int C) {
    const int h = H / 2, w = W / 2, G = C / 8;
    long long idx = (long long)blockIdx.x * TPB + threadIdx.x;
    if (idx >= (long long)B * h * w * G) return;
    const int q = (int)(idx / G), c = (int)(idx % G) * 8;
    const int b = q / (h * w), r = q - b * h * w, yy = r / w, xx = r - yy * w;
    float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
    for (int d = 0; d < 4; d++) {
        float f[8];
        unpack8(*(const uint4*)(x + ((size_t)(b * H + 2 * yy + d / 2) * W + 2 * xx + d % 2) * C + c), f);
#pragma unroll
        for (int j = 0; j < 8; j++) acc[j] += f[j];
    }
#pragma unroll
    for (int j = 0; j < 8; j++) acc[j] *= 0.25f;
    *(uint4*)(y + (size_t)q * C + c) = pack8(acc);
}

// dx[B, H, W, C] (+)= dy[B, H/2, W/2, C] / 4 at each of the four children
__global__ void k_pool2_bwd(const bf* __restrict__ dy, bf* __restrict__ dx, int B, int H, int W, int C, int accumulate) {
    const int h = H / 2, w = W / 2, G = C / 8;
    long long idx = (long long)blockIdx.x * TPB + threadIdx.x;
    if (idx >= (long long)B * H * W * G) return;
    const int p = (int)(idx / G), c = (int)(idx % G) * 8;
    const int b = p / (H * W), r = p - b * H * W, yy = r / W, xx = r - yy * W;
    float f[8];
    unpack8(*(const uint4*)(dy + ((size_t)(b * h + yy / 2) * w + xx / 2) * C + c), f);
#pragma unroll
    for (int j = 0; j < 8; j++) f[j] *= 0.25f;
    uint4* o = (uint4*)(dx + (size_t)p * C + c);
    if (accumulate) {
        float g[8];
        unpack8(*o, g);
#pragma unroll
        for (int j = 0; j < 8; j++) f[j] += g[j];
    }
    *o = pack8(f);
}

// nearest 2x upsampling of x[B, h, w, C] into channels [c0, c0 + C) of
// y[B, 2h, 2w, ldy] (the first part of a concatenation)
__global__ void k_up2(const bf* __restrict__ x, bf* __restrict__ y, int B, int h, int w, int C, int ldy, int c0) {
    const int H = 2 * h, W = 2 * w, G = C / 8;
    long long idx = (long long)blockIdx.x * TPB + threadIdx.x;
    if (idx >= (long long)B * H * W * G) return;
    const int p = (int)(idx / G), c = (int)(idx % G) * 8;
    const int b = p / (H * W), r = p - b * H * W, yy = r / W, xx = r - yy * W;
    *(uint4*)(y + (size_t)p * ldy + c0 + c) = *(const uint4*)(x + ((size_t)(b * h + yy / 2) * w + xx / 2) * C + c);
}

// dx[B, h, w, C] = sum of the four children's dy channels [c0, c0 + C)
__global__ void k_up2_bwd(const bf* __restrict__ dy, bf* __restrict__ dx, int B, int h, int w, int C, int ldy, int c0) {
    const int H = 2 * h, W = 2 * w, G = C / 8;
    long long idx = (long long)blockIdx.x * TPB + threadIdx.x;
    if (idx >= (long long)B * h * w * G) return;
    const int q = (int)(idx / G), c = (int)(idx % G) * 8;
    const int b = q / (h * w), r = q - b * h * w, yy = r / w, xx = r - yy * w;
    float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
    for (int d = 0; d < 4; d++) {
        float f[8];
        unpack8(*(const uint4*)(dy + ((size_t)(b * H + 2 * yy + d / 2) * W + 2 * xx + d % 2) * ldy + c0 + c), f);
#pragma unroll
        for (int j = 0; j < 8; j++) acc[j] += f[j];
    }
    *(uint4*)(dx + (size_t)q * C + c) = pack8(acc);
}

// copy x[P][C] into channels [c0, c0 + C) of y[P][ldy] (or back: reverse=1
// copies y's channels into x, optionally adding)
__global__ void k_chan_copy(bf* __restrict__ x, bf* __restrict__ y, long long P, int C, int ldy, int c0, int reverse,
                            int accumulate) {
    const int G = C / 8;
    long long idx = (long long)blockIdx.x * TPB + threadIdx.x;
    if (idx >= P * G) return;
    const long long p = idx / G;
    const int c = (int)(idx % G) * 8;
    uint4* xp = (uint4*)(x + (size_t)p * C + c);
    uint4* yp = (uint4*)(y + (size_t)p * ldy + c0 + c);
    if (!reverse) { *yp = *xp; return; }
    if (!accumulate) { *xp = *yp; return; }
    float a[8], b[8];
    unpack8(*xp, a);
    unpack8(*yp, b);
#pragma unroll
    for (int j = 0; j < 8; j++) a[j] += b[j];
    *xp = pack8(a);
}

// mean squared error over P pixels x nc channels of pred[P][ldp] (f32) and
// target[P][nc] (f32); dpred[P][ldg] (bf16) = 2 (pred - target) / (P nc),
// zero in the padding channels; loss[0] += sum of squares / (P nc)
// one thread per pixel and 8-wide group of gradient columns (ldg % 8 == 0):
// one 16-byte store of the bf16 gradient, the squared errors summed per
// block and added to *loss once per block
__global__ void k_mse(const float* __restrict__ pred, const float* __restrict__ tgt, bf* __restrict__ dpred,
                      float* __restrict__ loss, int P, int nc, int ldp, int ldg, float scale) {
    __shared__ float red[TPB / 32];
    float s = 0.0f;
    const int G = ldg / 8;
    const int n = P * G;   // < 2^31 (checked by the host)
    for (int idx = blockIdx.x * TPB + threadIdx.x; idx < n; idx += gridDim.x * TPB) {
        const int p = idx / G, c0 = (idx - p * G) * 8;
        __align__(16) bf g[8];
#pragma unroll
        for (int e = 0; e < 8; e++) {
            const int c = c0 + e;
            float v = 0.0f;
            if (c < nc) {
                const float d = pred[(size_t)p * ldp + c] - tgt[(size_t)p * nc + c];
                s += d * d;
                v = 2.0f * d * scale;
            }
            g[e] = __float2bfloat16(v);
        }
        *(uint4*)(dpred + (size_t)p * ldg + c0) = *(const uint4*)g;
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        float t = 0.0f;
        for (int w = 0; w < TPB / 32; w++) t += red[w];
        atomicAdd(loss, t * scale);
    }
}

// Adam on fp32 master weights p (n values), keeping a bf16 copy pb (same
// layout) for the GEMMs; lr_t is the bias-corrected step size.
__global__ void k_adam(float* __restrict__ p, bf* __restrict__ pb, const float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, long long n, float lr_t, float b1, float b2, float eps, float vcorr) {
    long long i = (long long)blockIdx.x * TPB + threadIdx.x;
    if (i >= n) return;
    float gi = g[i];
    float mi = b1 * m[i] + (1.0f - b1) * gi;
    float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    float pi = p[i] - lr_t * mi / (sqrtf(vi * vcorr) + eps);
    p[i] = pi;
    pb[i] = __float2bfloat16(pi);
}

// f32 -> bf16 (n values) and bf16 -> f32
__global__ void k_to_bf16(const float* __restrict__ a, bf* __restrict__ b, long long n) {
    long long i = (long long)blockIdx.x * TPB + threadIdx.x;
    if (i < n) b[i] = __float2bfloat16(a[i]);
}

// x[p][c] = bf16((planes[c][p] - mean[c]) * inv_std[c]) (a NULL plane is 0)
__global__ void k_encode(const float* const* __restrict__ planes, int nc, const float* __restrict__ mean,
                         const float* __restrict__ inv_std, bf* __restrict__ x, long long P) {
    long long idx = (long long)blockIdx.x * TPB + threadIdx.x;
    if (idx >= P * nc) return;
    const long long p = idx / nc;
    const int c = (int)(idx % nc);
    const float* pl = planes[c];
    float v = pl ? (pl[p] - mean[c]) * inv_std[c] : 0.0f;
    x[idx] = __float2bfloat16(v);
}

// dst[c][p] = hold[c][p] + out[p][c] * ys[c] + ym[c]
__global__ void k_decode(const float* __restrict__ out, int ldo, const float* const* __restrict__ hold,
                         const float* __restrict__ ym, const float* __restrict__ ys, float* const* __restrict__ dst,
                         int nc, long long P) {
    long long idx = (long long)blockIdx.x * TPB + threadIdx.x;
    if (idx >= P * nc) return;
    const int c = (int)(idx / P);
    const long long p = idx % P;
    dst[c][p] = hold[c][p] + out[p * ldo + c] * ys[c] + ym[c];
}

// Network input of several images of different sizes padded to one Hp x Wp:
// image b (nx = dims[2b], ny = dims[2b+1] <= Hp, Wp) from its planes
// planes[b*nc + c] (a NULL plane is the constant cval[b*nc + c], or 0);
// pixels beyond the image repeat its last column / row.
__global__ void k_encode_batch(const float* const* __restrict__ planes, int nc, const int* __restrict__ dims,
                               const float* __restrict__ cval, const float* __restrict__ mean,
                               const float* __restrict__ inv_std, bf* __restrict__ x, int nimg, int Hp, int Wp) {
    const long long idx = (long long)blockIdx.x * TPB + threadIdx.x;
    const long long total = (long long)nimg * Hp * Wp * nc;
    if (idx >= total) return;
    const int c = (int)(idx % nc);
    const long long pix = idx / nc;
    const int xw = (int)(pix % Wp);
    const long long r = pix / Wp;
    const int yh = (int)(r % Hp);
    const int b = (int)(r / Hp);
    const int nx = dims[2 * b], ny = dims[2 * b + 1];
    const float* pl = planes[(long long)b * nc + c];
    const int xs = min(xw, nx - 1), ys = min(yh, ny - 1);
    float v = 0.0f;
    if (pl) v = (pl[xs + (long long)ys * nx] - mean[c]) * inv_std[c];
    else if (cval) v = (cval[(long long)b * nc + c] - mean[c]) * inv_std[c];
    x[idx] = __float2bfloat16(v);
}

// Network output of a padded batch back to each image's planes:
// dst[b*nc + c][p] = hold[b*nc + c][p] + out[b][y][x][c] * ys[c] + ym[c]
// for the image's own pixels, and dst0[b*nc + c][p] = hold[...][p] when dst0
// is given (the fields the prediction starts from, kept).
__global__ void k_decode_batch(const float* __restrict__ out, int ldo, const float* const* __restrict__ hold,
                               const float* __restrict__ ym, const float* __restrict__ ysd,
                               float* const* __restrict__ dst, float* const* __restrict__ dst0,
                               const int* __restrict__ dims, int nc, int nimg, int Hp, int Wp) {
    const long long idx = (long long)blockIdx.x * TPB + threadIdx.x;
    const long long total = (long long)nimg * Hp * Wp * nc;
    if (idx >= total) return;
    const int c = (int)(idx % nc);
    const long long pix = idx / nc;
    const int xw = (int)(pix % Wp);
    const long long r = pix / Wp;
    const int yh = (int)(r % Hp);
    const int b = (int)(r / Hp);
    const int nx = dims[2 * b], ny = dims[2 * b + 1];
    if (xw >= nx || yh >= ny) return;
    const long long p = xw + (long long)yh * nx;
    const long long k = (long long)b * nc + c;
    const float h = hold[k][p];
    dst[k][p] = h + out[pix * ldo + c] * ysd[c] + ym[c];
    if (dst0) dst0[k][p] = h;
}

// dst[c][p] = src[c][p] (device arrays of nc plane pointers)
__global__ void k_copy_planes(const float* const* __restrict__ src, float* const* __restrict__ dst, int nc,
                              long long P) {
    long long idx = (long long)blockIdx.x * TPB + threadIdx.x;
    if (idx >= P * nc) return;
    const int c = (int)(idx / P);
    const long long p = idx % P;
    dst[c][p] = src[c][p];
}

}  // namespace nn
}  // namespace xbg

using namespace xbg::nn;

// wf[c][tap*cd + n] = w[n][(8-tap)*cin + c]; zero for k >= 9*cd
__global__ void k_flip3x3(const bf* __restrict__ w, int ldw, int cin, int cd, bf* __restrict__ wf, int ldf) {
    const long long idx = (long long)blockIdx.x * TPB + threadIdx.x;
    if (idx >= (long long)cin * ldf) return;
    const int c = (int)(idx / ldf), k = (int)(idx - (long long)c * ldf);
    bf v = __float2bfloat16(0.0f);
    if (k < 9 * cd) {
        const int tap = k / cd, n = k - tap * cd;
        v = w[(size_t)n * ldw + (8 - tap) * cin + c];
    }
    wf[idx] = v;
}

// dst[b][r][q] = src[s_b][y_b + r][x_b + q] for crop x crop pixels of `wpp`
// 4-byte words each (idx: s, y, x per crop); one thread per word
__global__ void k_gather_crops(const unsigned* __restrict__ src, unsigned* __restrict__ dst,
                               const int* __restrict__ idx, int ny, int nx, int crop, int wpp, long long n) {
    const long long t = (long long)blockIdx.x * TPB + threadIdx.x;
    if (t >= n) return;
    const long long row = (long long)crop * wpp;        // words of one crop row
    const long long per = row * crop;                   // words of one crop
    const int b = (int)(t / per);
    const long long r = t - (long long)b * per;
    const int y = (int)(r / row);
    const long long w = r - (long long)y * row;
    const int s = idx[3 * b], y0 = idx[3 * b + 1], x0 = idx[3 * b + 2];
    dst[t] = src[(((long long)s * ny + y0 + y) * nx + x0) * wpp + w];
}

#define NN_LAUNCH(n) if ((n) <= 0) return XBG_OK; cudaStream_t st_ = (cudaStream_t)stream
#define NN_DONE return cudaGetLastError() == cudaSuccess ? XBG_OK : XBG_ERR_CUDA

extern "C" {

int xbg_nn_im2col3x3(const void* x, void* col, int B, int H, int W, int C, int Kp, int Mpad, void* stream) {
    if (!x || !col || B < 1 || H < 1 || W < 1 || C < 8 || (C % 8) || (Kp % 64) || Kp < 9 * C || Mpad < B * H * W)
        return XBG_ERR_ARG;
    long long n = (long long)Mpad * (Kp / 8);
    NN_LAUNCH(n);
    k_im2col<<<blocks_for(n), TPB, 0, st_>>>((const bf*)x, (bf*)col, B, H, W, C, Kp, Mpad);
    NN_DONE;
}
int xbg_nn_col2im3x3(const void* dcol, void* dx, int B, int H, int W, int C, int Kp, int accumulate, void* stream) {
    if (!dcol || !dx || B < 1 || H < 1 || W < 1 || C < 8 || (C % 8) || Kp < 9 * C) return XBG_ERR_ARG;
    long long n = (long long)B * H * W * (C / 8);
    NN_LAUNCH(n);
    k_col2im<<<blocks_for(n), TPB, 0, st_>>>((const bf*)dcol, (bf*)dx, B, H, W, C, Kp, accumulate);
    NN_DONE;
}
int xbg_nn_conv3x3_flip(const void* w, int ldw, int cin, int cd, void* wf, int ldf, void* stream) {
    if (!w || !wf || cin < 1 || cd < 1 || ldw < 9 * cin || ldf < 9 * cd) return XBG_ERR_ARG;
    long long n = (long long)cin * ldf;
    NN_LAUNCH(n);
    k_flip3x3<<<blocks_for(n), TPB, 0, st_>>>((const bf*)w, ldw, cin, cd, (bf*)wf, ldf);
    NN_DONE;
}
int xbg_nn_gather_crops(const void* src, void* dst, const int* idx, int B, int ny, int nx, int crop,
                        int bytes_per_px, void* stream) {
    if (!src || !dst || !idx || B < 1 || crop < 1 || crop > ny || crop > nx || bytes_per_px < 4 ||
        (bytes_per_px % 4) || (((uintptr_t)src | (uintptr_t)dst) & 3))
        return XBG_ERR_ARG;
    const long long n = (long long)B * crop * crop * (bytes_per_px / 4);
    NN_LAUNCH(n);
    k_gather_crops<<<blocks_for(n), TPB, 0, st_>>>((const unsigned*)src, (unsigned*)dst, idx, ny, nx, crop,
                                                   bytes_per_px / 4, n);
    NN_DONE;
}
int xbg_nn_transpose(const void* src, void* dst, int R, int Cc, int lds, int ldd, void* stream) {
    if (!src || !dst || R < 1 || Cc < 1 || lds < Cc || ldd < R) return XBG_ERR_ARG;
    cudaStream_t st_ = (cudaStream_t)stream;
    dim3 g((R + 31) / 32, (Cc + 31) / 32), b(32, 8);
    k_transpose<<<g, b, 0, st_>>>((const bf*)src, (bf*)dst, R, Cc, lds, ldd);
    NN_DONE;
}
int xbg_nn_relu_bwd(const void* dy, const void* y, void* dx, long long n, void* stream) {
    if (!dy || !y || !dx || n < 0 || (n % 8)) return XBG_ERR_ARG;
    NN_LAUNCH(n / 8);
    k_relu_bwd<<<blocks_for(n / 8), TPB, 0, st_>>>((const bf*)dy, (const bf*)y, (bf*)dx, n / 8);
    NN_DONE;
}
int xbg_nn_bias_grad(const void* dy, float* db, int P, int N, int ld, void* stream) {
    if (!dy || !db || P < 1 || N < 1 || N > 256 || ld < N) return XBG_ERR_ARG;
    cudaStream_t st_ = (cudaStream_t)stream;
    k_bias_grad<<<(P + 255) / 256, TPB, 0, st_>>>((const bf*)dy, db, P, N, ld);
    NN_DONE;
}
int xbg_nn_pool2(const void* x, void* y, int B, int H, int W, int C, void* stream) {
    if (!x || !y || B < 1 || H < 2 || W < 2 || (H % 2) || (W % 2) || C < 8 || (C % 8)) return XBG_ERR_ARG;
    long long n = (long long)B * (H / 2) * (W / 2) * (C / 8);
    NN_LAUNCH(n);
    k_pool2<<<blocks_for(n), TPB, 0, st_>>>((const bf*)x, (bf*)y, B, H, W, C);
    NN_DONE;
}
int xbg_nn_pool2_bwd(const void* dy, void* dx, int B, int H, int W, int C, int accumulate, void* stream) {
    if (!dy || !dx || B < 1 || H < 2 || W < 2 || (H % 2) || (W % 2) || C < 8 || (C % 8)) return XBG_ERR_ARG;
    long long n = (long long)B * H * W * (C / 8);
    NN_LAUNCH(n);
    k_pool2_bwd<<<blocks_for(n), TPB, 0, st_>>>((const bf*)dy, (bf*)dx, B, H, W, C, accumulate);
    NN_DONE;
}
int xbg_nn_up2(const void* x, void* y, int B, int h, int w, int C, int ldy, int c0, void* stream) {
    if (!x || !y || B < 1 || h < 1 || w < 1 || C < 8 || (C % 8) || (c0 % 8) || (ldy % 8) || c0 + C > ldy)
        return XBG_ERR_ARG;
    long long n = (long long)B * 4 * h * w * (C / 8);
    NN_LAUNCH(n);
    k_up2<<<blocks_for(n), TPB, 0, st_>>>((const bf*)x, (bf*)y, B, h, w, C, ldy, c0);
    NN_DONE;
}
int xbg_nn_up2_bwd(const void* dy, void* dx, int B, int h, int w, int C, int ldy, int c0, void* stream) {
    if (!dy || !dx || B < 1 || h < 1 || w < 1 || C < 8 || (C % 8) || (c0 % 8) || (ldy % 8) || c0 + C > ldy)
        return XBG_ERR_ARG;
    long long n = (long long)B * h * w * (C / 8);
    NN_LAUNCH(n);
    k_up2_bwd<<<blocks_for(n), TPB, 0, st_>>>((const bf*)dy, (bf*)dx, B, h, w, C, ldy, c0);
    NN_DONE;
}
int xbg_nn_chan_copy(void* x, void* y, long long P, int C, int ldy, int c0, int reverse, int accumulate, void* stream) {
    if (!x || !y || P < 1 || C < 8 || (C % 8) || (c0 % 8) || (ldy % 8) || c0 + C > ldy) return XBG_ERR_ARG;
    long long n = P * (C / 8);
    NN_LAUNCH(n);
    k_chan_copy<<<blocks_for(n), TPB, 0, st_>>>((bf*)x, (bf*)y, P, C, ldy, c0, reverse, accumulate);
    NN_DONE;
}
int xbg_nn_mse(const float* pred, const float* tgt, void* dpred, float* loss, int P, int nc, int ldp, int ldg,
               void* stream) {
    if (!pred || !tgt || !dpred || !loss || P < 1 || nc < 1 || ldp < nc || ldg < nc || (ldg % 8) ||
        ((uintptr_t)dpred & 15) || (long long)P * (ldg / 8) > 0x7fffffffLL - 1184LL * TPB)
        return XBG_ERR_ARG;
    long long n = (long long)P * (ldg / 8);
    NN_LAUNCH(n);
    // grid-stride over a few blocks per SM: one atomic add of the loss per block
    const unsigned nb = (unsigned)(blocks_for(n) < 1184 ? blocks_for(n) : 1184);
    k_mse<<<nb, TPB, 0, st_>>>(pred, tgt, (bf*)dpred, loss, P, nc, ldp, ldg, 1.0f / ((float)P * nc));
    NN_DONE;
}
int xbg_nn_adam(float* p, void* pb, const float* g, float* m, float* v, long long n, float lr, float b1, float b2,
                float eps, int step, void* stream) {
    if (!p || !pb || !g || !m || !v || n < 0 || step < 1) return XBG_ERR_ARG;
    NN_LAUNCH(n);
    float bc1 = 1.0f - powf(b1, (float)step), bc2 = 1.0f - powf(b2, (float)step);
    k_adam<<<blocks_for(n), TPB, 0, st_>>>(p, (bf*)pb, g, m, v, n, lr / bc1, b1, b2, eps, 1.0f / bc2);
    NN_DONE;
}
int xbg_nn_encode(const float* const* planes, int nc, const float* mean, const float* inv_std, void* x, long long P,
                  void* stream) {
    if (!planes || !mean || !inv_std || !x || nc < 1 || P < 1) return XBG_ERR_ARG;
    NN_LAUNCH(P * nc);
    k_encode<<<blocks_for(P * nc), TPB, 0, st_>>>(planes, nc, mean, inv_std, (bf*)x, P);
    NN_DONE;
}
int xbg_nn_decode(const float* out, int ldo, const float* const* hold, const float* ym, const float* ys,
                  float* const* dst, int nc, long long P, void* stream) {
    if (!out || !hold || !ym || !ys || !dst || nc < 1 || ldo < nc || P < 1) return XBG_ERR_ARG;
    NN_LAUNCH(P * nc);
    k_decode<<<blocks_for(P * nc), TPB, 0, st_>>>(out, ldo, hold, ym, ys, dst, nc, P);
    NN_DONE;
}
int xbg_nn_encode_batch(const float* const* planes, int nc, const int* dims, const float* cval, const float* mean,
                        const float* inv_std, void* x, int nimg, int Hp, int Wp, void* stream) {
    if (!planes || !dims || !mean || !inv_std || !x || nc < 1 || nimg < 1 || Hp < 1 || Wp < 1) return XBG_ERR_ARG;
    const long long n = (long long)nimg * Hp * Wp * nc;
    NN_LAUNCH(n);
    k_encode_batch<<<blocks_for(n), TPB, 0, st_>>>(planes, nc, dims, cval, mean, inv_std, (bf*)x, nimg, Hp, Wp);
    NN_DONE;
}
int xbg_nn_decode_batch(const float* out, int ldo, const float* const* hold, const float* ym, const float* ys,
                        float* const* dst, float* const* dst0, const int* dims, int nc, int nimg, int Hp, int Wp,
                        void* stream) {
    if (!out || !hold || !ym || !ys || !dst || !dims || nc < 1 || ldo < nc || nimg < 1 || Hp < 1 || Wp < 1)
        return XBG_ERR_ARG;
    const long long n = (long long)nimg * Hp * Wp * nc;
    NN_LAUNCH(n);
    k_decode_batch<<<blocks_for(n), TPB, 0, st_>>>(out, ldo, hold, ym, ys, dst, dst0, dims, nc, nimg, Hp, Wp);
    NN_DONE;
}
int xbg_nn_copy_planes(const float* const* src, float* const* dst, int nc, long long P, void* stream) {
    if (!src || !dst || nc < 1 || P < 1) return XBG_ERR_ARG;
    NN_LAUNCH(P * nc);
    k_copy_planes<<<blocks_for(P * nc), TPB, 0, st_>>>(src, dst, nc, P);
    NN_DONE;
}
int xbg_nn_to_bf16(const float* a, void* b, long long n, void* stream) {
    if (!a || !b || n < 0) return XBG_ERR_ARG;
    NN_LAUNCH(n);
    k_to_bf16<<<blocks_for(n), TPB, 0, st_>>>(a, (bf*)b, n);
    NN_DONE;
}

}  // extern "C"
