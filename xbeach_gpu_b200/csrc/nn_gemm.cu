// nn_gemm.cu -- the tensor-core GEMM of the wave surrogate (5th-generation
// tensor cores, tcgen05, accumulators in tensor memory).
//
//   C[M x N] = act(A[M x K] . B[N x K]^T + bias[N])
//
// A and B are bf16, row-major with K contiguous ("K-major"); C is fp32 or bf16
// row-major; the products accumulate in fp32.  One CTA computes a 128 x BN
// tile (BN = N, 16..256, a multiple of 16; M is padded by the caller to a
// multiple of 128 and K to a multiple of 64).
//
// Per 64-wide K chunk: all 256 threads copy the A and B chunk into shared
// memory (cp.async, 16 B) in the canonical K-major 128-byte-swizzle layout
// (row pitch 128 B, the 16-byte chunk index XOR the row within its 8-row
// group, 1024-B aligned tiles), fence the async proxy and sync; one thread
// issues four tcgen05.mma of 128 x BN x 16 (smem descriptors advanced by
// 32 B) and commits them to the stage's mbarrier.  Three stages: the copies
// of chunk k+2 are in flight while the MMAs of chunk k run; a stage is
// refilled once the commit of its last MMAs has arrived.  The epilogue waits for the last
// commit, reads the accumulators with tcgen05.ld (warp w reads TMEM lanes
// 32*(w%4).. and half of the columns), adds the bias, applies ReLU and
// stores.  Every mbarrier wait is bounded: on time-out the kernel records an
// error code and leaves (the host reads it).
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include <cstdint>

#include "../../include/xbg.h"
#include "../../include/xbg_nn.h"

namespace xbg {
namespace nn {

constexpr int GM = 128;          // rows of a CTA tile (TMEM lanes)
constexpr int GK = 64;           // K chunk: 64 bf16 = one 128-B swizzle row
constexpr int GSTAGES = 3;
constexpr unsigned WAIT_LIMIT = 1u << 22;   // try_wait polls before giving up
constexpr unsigned CHECK_WAIT_LIMIT = 4096; // polls of the time-out check (XBG_NN_CHECK_TIMEOUT)

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void cp16(unsigned dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(src));
}

// K-major, 128-B swizzle shared-memory matrix descriptor (start address and
// strides in 16-B units; SBO = 1024 B between 8-row groups; version 1).
__device__ __forceinline__ uint64_t sw128_desc(unsigned saddr) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);
    d |= (uint64_t)1 << 16;                 // LBO (unused with this swizzle)
    d |= (uint64_t)(1024 >> 4) << 32;       // SBO
    d |= (uint64_t)1 << 46;                 // descriptor version
    d |= (uint64_t)2 << 61;                 // SWIZZLE_128B
    return d;
}

// kind::f16 instruction descriptor: bf16 x bf16 -> f32, both K-major, M x N
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mbar_init(unsigned a, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(a), "r"(count));
}
// bounded wait for the phase with the given parity; false on time-out
__device__ __forceinline__ bool mbar_wait(unsigned a, unsigned parity, unsigned limit = WAIT_LIMIT) {
    for (unsigned it = 0; it < limit; it++) {
        unsigned ok;
        asm volatile(
            "{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\nselp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(ok)
            : "r"(a), "r"(parity)
            : "memory");
        if (ok) return true;
    }
    return false;
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

template <int BN>
__global__ void __launch_bounds__(256, 2) k_gemm_tc(const __nv_bfloat16* __restrict__ A,
                                                    const __nv_bfloat16* __restrict__ B,
                                                    const float* __restrict__ bias, void* C, int M, int N, int K,
                                                    int lda, int ldb, int ldc, int flags, int* err) {
    constexpr int A_BYTES = GM * GK * 2;       // 16 KB
    constexpr int B_BYTES = BN * GK * 2;
    constexpr int STAGE = A_BYTES + B_BYTES;   // multiple of 1024
    constexpr int TCOLS = BN <= 32 ? 32 : (BN <= 64 ? 64 : (BN <= 128 ? 128 : 256));
    extern __shared__ unsigned char smem_raw[];
    __shared__ __align__(8) unsigned long long mbar[GSTAGES + 1];   // + the time-out check's barrier
    __shared__ unsigned tmem_slot;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.x * GM;
    // split-K: this CTA reduces K chunks [kb, ke) (whole K unless gridDim.y > 1)
    const int nk_all = K / GK;
    const int per = (nk_all + gridDim.y - 1) / gridDim.y;
    const int kb = blockIdx.y * per, ke = min(nk_all, kb + per);
    // 1024-B aligned stage buffers
    const unsigned base = (smem_u32(smem_raw) + 1023u) & ~1023u;
    unsigned char* gbase = smem_raw + (base - smem_u32(smem_raw));

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(&tmem_slot)),
                     "r"(TCOLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
    }
    if (tid == 0) {
        for (int s = 0; s <= GSTAGES; s++) mbar_init(smem_u32(&mbar[s]), 1);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const unsigned tmem = tmem_slot;
    const uint32_t idesc = idesc_bf16(GM, BN);
    bool ok = true;
    if (flags & XBG_NN_CHECK_TIMEOUT) {
        // check of the time-out exit: a short bounded wait on a barrier that
        // nothing arrives on runs out, and the CTA leaves the way a stalled
        // pipeline does (nothing issued, error recorded, tensor memory freed)
        ok = __syncthreads_and(mbar_wait(smem_u32(&mbar[GSTAGES]), 0, CHECK_WAIT_LIMIT)) != 0;
    }
    const int nk = ok ? max(0, ke - kb) : 0;
    int issued = 0;   // chunks whose MMAs were committed
    // copy K chunk kc (of this CTA's range) into stage s
    auto load = [&](int kc, int s) {
        const unsigned sa = base + s * STAGE, sb = sa + A_BYTES;
        const int k0 = (kb + kc) * GK;
        for (int q = tid; q < GM * 8; q += 256) {   // A: 128 rows x 8 chunks
            int r = q >> 3, c = q & 7;
            int m = m0 + r;
            unsigned dst = sa + r * 128 + ((c ^ (r & 7)) << 4);
            if (m < M) cp16(dst, A + (size_t)m * lda + k0 + c * 8);
            else *(uint4*)(gbase + (dst - base)) = make_uint4(0, 0, 0, 0);
        }
        for (int q = tid; q < BN * 8; q += 256) {   // B: BN rows x 8 chunks
            int r = q >> 3, c = q & 7;
            unsigned dst = sb + r * 128 + ((c ^ (r & 7)) << 4);
            if (r < N) cp16(dst, B + (size_t)r * ldb + k0 + c * 8);
            else *(uint4*)(gbase + (dst - base)) = make_uint4(0, 0, 0, 0);
        }
    };
    // pipeline as in k_conv_tc: copies of chunk kc+2 overlap the MMAs of chunk kc
    for (int kc = 0; kc < GSTAGES - 1; kc++) {
        if (kc < nk) load(kc, kc);
        asm volatile("cp.async.commit_group;\n" ::: "memory");
    }
    for (int kc = 0; kc < nk; kc++) {
        const int s = kc % GSTAGES;
        const int kn = kc + GSTAGES - 1;
        if (kn < nk) {
            if (kc >= 1) {   // the MMAs of chunk kc-1 read the stage chunk kn goes to
                const bool w = mbar_wait(smem_u32(&mbar[(kc - 1) % GSTAGES]), ((kc - 1) / GSTAGES) & 1);
                if (!__syncthreads_and(w)) { ok = false; break; }
            }
            load(kn, kn % GSTAGES);
        }
        asm volatile("cp.async.commit_group;\n" ::: "memory");
        asm volatile("cp.async.wait_group %0;\n" ::"n"(GSTAGES - 1) : "memory");   // chunk kc has landed
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            tc_fence_after();
            const unsigned sa = base + s * STAGE, sb = sa + A_BYTES;
            const uint64_t da = sw128_desc(sa), db = sw128_desc(sb);
#pragma unroll
            for (int j = 0; j < GK / 16; j++) {
                const unsigned acc = (kc > 0 || j > 0) ? 1u : 0u;
                asm volatile(
                    "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
                    "l"(da + (uint64_t)(2 * j)), "l"(db + (uint64_t)(2 * j)), "r"(idesc), "r"(acc));
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                             smem_u32(&mbar[s]))
                         : "memory");
        }
        issued = kc + 1;
    }
    asm volatile("cp.async.wait_all;\n" ::: "memory");
    if (ok && nk > 0) ok = mbar_wait(smem_u32(&mbar[(nk - 1) % GSTAGES]), ((nk - 1) / GSTAGES) & 1);
    ok = __syncthreads_and(ok) != 0;   // the TMEM loads below are warp-collective
    if (!ok && issued > 0)   // leaving early: let the committed MMAs finish (bounded) before TMEM is freed
        mbar_wait(smem_u32(&mbar[(issued - 1) % GSTAGES]), ((issued - 1) / GSTAGES) & 1);
    tc_fence_after();

    if (ok) {   // epilogue: warp w -> lanes 32*(w%4).., column half w/4
        const int q = warp & 3, h = warp >> 2;
        const int row = m0 + q * 32 + lane;
        const int half = BN / 2;
        for (int c0 = h * half; c0 < (h + 1) * half; c0 += 8) {
            unsigned r[8];
            const unsigned taddr = tmem + ((unsigned)(q * 32) << 16) + (unsigned)c0;
            asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];\n"
                         : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
                           "=r"(r[7])
                         : "r"(taddr));
            asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
            if (row < M) {
#pragma unroll
                for (int j = 0; j < 8; j++) {
                    const int n = c0 + j;
                    if (n >= N) break;
                    float v = nk > 0 ? __uint_as_float(r[j]) : 0.0f;
                    if (flags & XBG_NN_ATOMIC) {   // split-K partial: add into f32 C
                        atomicAdd((float*)C + (size_t)row * ldc + n, v);
                        continue;
                    }
                    if (bias) v += bias[n];
                    if (flags & XBG_NN_RELU) v = fmaxf(v, 0.0f);
                    if (flags & XBG_NN_OUT_BF16) ((__nv_bfloat16*)C)[(size_t)row * ldc + n] = __float2bfloat16(v);
                    else ((float*)C)[(size_t)row * ldc + n] = v;
                }
            }
        }
    } else if (tid == 0) {
        atomicExch(err, XBG_ERR_TIMEOUT);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(TCOLS));
}

template <int BN>
int gemm_launch(const void* A, const void* B, const float* bias, void* C, int M, int N, int K, int lda, int ldb,
                int ldc, int flags, int ksplit, int* err, cudaStream_t st) {
    constexpr int STAGE = GM * GK * 2 + BN * GK * 2;
    const size_t smem = (size_t)GSTAGES * STAGE + 1024;
    static bool attr = false;   // per process; the attribute is per function
    if (!attr) {
        if (cudaFuncSetAttribute(k_gemm_tc<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
            return XBG_ERR_CUDA;
        attr = true;
    }
    dim3 grid((M + GM - 1) / GM, ksplit);
    k_gemm_tc<BN><<<grid, 256, smem, st>>>((const __nv_bfloat16*)A, (const __nv_bfloat16*)B, bias, C, M, N, K, lda,
                                           ldb, ldc, flags, err);
    return cudaGetLastError() == cudaSuccess ? XBG_OK : XBG_ERR_CUDA;
}

// ------------------------------------------------------------------------
// 3x3 convolution as an implicit GEMM: y[p][n] = act(sum over tap, c of
// x[b, y+dy, x+dx, c] w[n][tap*cin + c] + bias[n]), the A operand (one row
// per output pixel, K = tap*cin + c) gathered from the NHWC input straight
// into the swizzled shared-memory tile, 16 bytes (8 channels of one tap) per
// copy, zero outside the image and beyond tap 8.  Three cp.async stages: the
// copies of chunk k+2 overlap the MMAs of chunk k; each stage is reused
// after its MMAs' commit arrives.  Several CTAs per SM (small tiles, little
// shared memory); the epilogue stores 8 channels per 16-byte write.
constexpr int CSTAGES = 3;

template <int BN>
__global__ void __launch_bounds__(256, 2) k_conv_tc(const __nv_bfloat16* __restrict__ X,
                                                    const __nv_bfloat16* __restrict__ Wt,
                                                    const float* __restrict__ bias, void* Y, int Bn, int H, int W,
                                                    int cin, int ldx, int N, int Kp, int ldw, int ldy, int flags,
                                                    int* err) {
    constexpr int A_BYTES = GM * GK * 2;
    constexpr int B_BYTES = BN * GK * 2;
    constexpr int STAGE = A_BYTES + B_BYTES;
    constexpr int TCOLS = BN <= 32 ? 32 : (BN <= 64 ? 64 : (BN <= 128 ? 128 : 256));
    extern __shared__ unsigned char smem_raw[];
    __shared__ __align__(8) unsigned long long mbar[CSTAGES];
    __shared__ unsigned tmem_slot;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int M = Bn * H * W;
    const int m0 = blockIdx.x * GM;
    const int nk = Kp / GK;
    const unsigned base = (smem_u32(smem_raw) + 1023u) & ~1023u;
    unsigned char* gbase = smem_raw + (base - smem_u32(smem_raw));
    // this thread's four A rows (pixels) and its 16-byte chunk within a row
    const int cch = tid & 7;
    int pb[4], py[4], px[4];
#pragma unroll
    for (int u = 0; u < 4; u++) {
        const int m = m0 + (tid >> 3) + 32 * u;
        if (m < M) {
            px[u] = m % W;
            const int t = m / W;
            py[u] = t % H;
            pb[u] = t / H;
        } else {
            pb[u] = -1; py[u] = 0; px[u] = 0;
        }
    }
    auto load = [&](int kc, int s) {
        const unsigned sa = base + s * STAGE, sb = sa + A_BYTES;
        const int k = kc * GK + cch * 8;
        const int tap = k / cin, ch = k - tap * cin;
        const int dy = tap / 3 - 1, dx = tap % 3 - 1;
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const int r = (tid >> 3) + 32 * u;
            const unsigned dst = sa + r * 128 + ((cch ^ (r & 7)) << 4);
            const int sy = py[u] + dy, sx = px[u] + dx;
            if (pb[u] >= 0 && tap < 9 && sy >= 0 && sy < H && sx >= 0 && sx < W)
                cp16(dst, X + ((size_t)(pb[u] * H + sy) * W + sx) * ldx + ch);
            else
                *(uint4*)(gbase + (dst - base)) = make_uint4(0, 0, 0, 0);
        }
        for (int q = tid; q < BN * 8; q += 256) {
            const int r = q >> 3, c = q & 7;
            const unsigned dst = sb + r * 128 + ((c ^ (r & 7)) << 4);
            if (r < N) cp16(dst, Wt + (size_t)r * ldw + kc * GK + c * 8);
            else *(uint4*)(gbase + (dst - base)) = make_uint4(0, 0, 0, 0);
        }
    };

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(&tmem_slot)),
                     "r"(TCOLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
    }
    if (tid == 0) {
        for (int s = 0; s < CSTAGES; s++) mbar_init(smem_u32(&mbar[s]), 1);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const unsigned tmem = tmem_slot;
    const uint32_t idesc = idesc_bf16(GM, BN);
    bool ok = true;
    int issued = 0;   // chunks whose MMAs were committed
    // prologue: chunks 0 .. CSTAGES-2 in flight
    for (int kc = 0; kc < CSTAGES - 1; kc++) {
        if (kc < nk) load(kc, kc);
        asm volatile("cp.async.commit_group;\n" ::: "memory");
    }
    for (int kc = 0; kc < nk; kc++) {
        const int s = kc % CSTAGES;
        // refill the stage of chunk kc-1 with chunk kc+CSTAGES-1 once its MMAs are done
        const int kn = kc + CSTAGES - 1;
        if (kn < nk) {
            if (kc >= 1) {
                const bool w = mbar_wait(smem_u32(&mbar[(kc - 1) % CSTAGES]), ((kc - 1) / CSTAGES) & 1);
                if (!__syncthreads_and(w)) { ok = false; break; }
            }
            load(kn, kn % CSTAGES);
        }
        asm volatile("cp.async.commit_group;\n" ::: "memory");
        asm volatile("cp.async.wait_group %0;\n" ::"n"(CSTAGES - 1) : "memory");   // chunk kc has landed
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            tc_fence_after();
            const unsigned sa = base + s * STAGE, sb = sa + A_BYTES;
            const uint64_t da = sw128_desc(sa), db = sw128_desc(sb);
#pragma unroll
            for (int j = 0; j < GK / 16; j++) {
                const unsigned acc = (kc > 0 || j > 0) ? 1u : 0u;
                asm volatile(
                    "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
                    "l"(da + (uint64_t)(2 * j)), "l"(db + (uint64_t)(2 * j)), "r"(idesc), "r"(acc));
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                             smem_u32(&mbar[s]))
                         : "memory");
        }
        issued = kc + 1;
    }
    asm volatile("cp.async.wait_all;\n" ::: "memory");
    if (ok && nk > 0) ok = mbar_wait(smem_u32(&mbar[(nk - 1) % CSTAGES]), ((nk - 1) / CSTAGES) & 1);
    ok = __syncthreads_and(ok) != 0;
    if (!ok && issued > 0)   // leaving early: let the committed MMAs finish (bounded) before TMEM is freed
        mbar_wait(smem_u32(&mbar[(issued - 1) % CSTAGES]), ((issued - 1) / CSTAGES) & 1);
    tc_fence_after();

    if (ok) {   // warp w -> TMEM lanes 32*(w%4).., column half w/4; 8 channels per store
        const int q = warp & 3, h = warp >> 2;
        const int row = m0 + q * 32 + lane;
        const int half = BN / 2;
        for (int c0 = h * half; c0 < (h + 1) * half; c0 += 8) {
            unsigned r[8];
            const unsigned taddr = tmem + ((unsigned)(q * 32) << 16) + (unsigned)c0;
            asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];\n"
                         : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
                           "=r"(r[7])
                         : "r"(taddr));
            asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
            if (row < M && c0 < N) {
                float v[8];
#pragma unroll
                for (int j = 0; j < 8; j++) {
                    v[j] = (nk > 0 ? __uint_as_float(r[j]) : 0.0f) + (bias ? bias[c0 + j] : 0.0f);
                    if (flags & XBG_NN_RELU) v[j] = fmaxf(v[j], 0.0f);
                }
                if (flags & XBG_NN_OUT_BF16) {
                    __align__(16) __nv_bfloat16 o[8];
#pragma unroll
                    for (int j = 0; j < 8; j++) o[j] = __float2bfloat16(v[j]);
                    *(uint4*)((__nv_bfloat16*)Y + (size_t)row * ldy + c0) = *(const uint4*)o;
                } else {
                    float* d = (float*)Y + (size_t)row * ldy + c0;
                    *(float4*)d = make_float4(v[0], v[1], v[2], v[3]);
                    *(float4*)(d + 4) = make_float4(v[4], v[5], v[6], v[7]);
                }
            }
        }
    } else if (tid == 0) {
        atomicExch(err, XBG_ERR_TIMEOUT);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(TCOLS));
}

// ------------------------------------------------------------------------
// The same convolution with the A operand moved by the tensor memory
// accelerator.  A CTA's 128 output pixels are R whole image rows of Wt
// pixels (Wt = W when W divides 128, else 128 pixels of one row), so for
// one tap the 128 input pixels it needs are one box [R][Wt] of the NHWC
// input shifted by (dy, dx); pixels outside the image arrive as zeros (the
// padding).  Each 64-wide K chunk is 64/WC boxes of WC channels (a tap's
// channel run, WC = 32, or 16 for 16-channel inputs), written by the copy
// engine in the WC*2-byte swizzled K-major layout the MMA reads, on the
// stage's "full" mbarrier; one elected thread issues them.  The weights
// (B) keep the cp.async copies.  Taps beyond the ninth (K padding) are
// zero-filled by the threads.  No multicast; the map covers this GPU's
// memory only.
template <int WC>
__host__ __device__ constexpr uint32_t sw_layout() { return WC == 32 ? 4u : 6u; }   // SWIZZLE_64B / SWIZZLE_32B

template <int WC>
__device__ __forceinline__ uint64_t swk_desc(unsigned saddr) {   // K-major, rows of WC*2 bytes
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);
    d |= (uint64_t)1 << 16;                          // LBO (unused with swizzling)
    d |= (uint64_t)((8 * WC * 2) >> 4) << 32;        // SBO: 8 rows
    d |= (uint64_t)1 << 46;
    d |= (uint64_t)sw_layout<WC>() << 61;
    return d;
}

template <int BN, int WC>
__global__ void __launch_bounds__(256, 2) k_conv_tma(const __grid_constant__ CUtensorMap xmap,
                                                     const __nv_bfloat16* __restrict__ Wt,
                                                     const float* __restrict__ bias, void* Y, int Bn, int H, int W,
                                                     int cin, int N, int Kp, int ldw, int ldy, int flags, int* err) {
    constexpr int NSUB = GK / WC;                 // boxes per K chunk
    constexpr int SUB_BYTES = GM * WC * 2;        // one box: 128 rows of WC channels
    constexpr int A_BYTES = GM * GK * 2;
    constexpr int B_BYTES = BN * GK * 2;
    constexpr int STAGE = A_BYTES + B_BYTES;
    constexpr int TCOLS = BN <= 32 ? 32 : (BN <= 64 ? 64 : (BN <= 128 ? 128 : 256));
    extern __shared__ unsigned char smem_raw[];
    __shared__ __align__(8) unsigned long long mbar[CSTAGES];    // MMAs of a stage done
    __shared__ __align__(8) unsigned long long full[CSTAGES];    // A boxes of a stage landed
    __shared__ unsigned tmem_slot;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int M = Bn * H * W;
    const int m0 = blockIdx.x * GM;
    const int nk = Kp / GK;
    const unsigned base = (smem_u32(smem_raw) + 1023u) & ~1023u;
    unsigned char* gbase = smem_raw + (base - smem_u32(smem_raw));
    // the tile's first pixel
    const int HW = H * W;
    const int tb = m0 / HW, rem = m0 - tb * HW;
    const int ty0 = rem / W, tx0 = rem - ty0 * W;
    auto load = [&](int kc, int s) {   // all threads: zero boxes, weights; thread 0: the A boxes
        const unsigned sa = base + s * STAGE, sb = sa + A_BYTES;
        int nbox = 0;
#pragma unroll
        for (int u = 0; u < NSUB; u++) {
            const int k0 = kc * GK + u * WC;
            if (k0 / cin >= 9) {   // K padding: zeros
                for (int q = tid; q < SUB_BYTES / 16; q += 256)
                    *(uint4*)(gbase + (sa + u * SUB_BYTES - base) + q * 16) = make_uint4(0, 0, 0, 0);
            } else {
                nbox++;
            }
        }
        if (tid == 0) {
            const unsigned fb = smem_u32(&full[s]);
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(fb),
                         "r"((unsigned)(nbox * SUB_BYTES))
                         : "memory");
#pragma unroll
            for (int u = 0; u < NSUB; u++) {
                const int k0 = kc * GK + u * WC;
                const int tap = k0 / cin;
                if (tap >= 9) continue;
                const int c0 = k0 - tap * cin;
                const int dy = tap / 3 - 1, dx = tap % 3 - 1;
                asm volatile(
                    "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, "
                    "%3, %4, %5}], [%6];\n" ::"r"(sa + u * SUB_BYTES),
                    "l"((unsigned long long)&xmap), "r"(c0), "r"(tx0 + dx), "r"(ty0 + dy), "r"(tb), "r"(fb)
                    : "memory");
            }
        }
        for (int q = tid; q < BN * 8; q += 256) {
            const int r = q >> 3, c = q & 7;
            const unsigned dst = sb + r * 128 + ((c ^ (r & 7)) << 4);
            if (r < N) cp16(dst, Wt + (size_t)r * ldw + kc * GK + c * 8);
            else *(uint4*)(gbase + (dst - base)) = make_uint4(0, 0, 0, 0);
        }
    };

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(&tmem_slot)),
                     "r"(TCOLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
    }
    if (tid == 0) {
        for (int s = 0; s < CSTAGES; s++) {
            mbar_init(smem_u32(&mbar[s]), 1);
            mbar_init(smem_u32(&full[s]), 1);
        }
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const unsigned tmem = tmem_slot;
    const uint32_t idesc = idesc_bf16(GM, BN);
    bool ok = true;
    int issued = 0;   // chunks whose MMAs were committed
    int loaded = 0;   // chunks whose boxes were issued
    for (int kc = 0; kc < CSTAGES - 1; kc++) {
        if (kc < nk) { load(kc, kc); loaded = kc + 1; }
        asm volatile("cp.async.commit_group;\n" ::: "memory");
    }
    for (int kc = 0; kc < nk; kc++) {
        const int s = kc % CSTAGES;
        const int kn = kc + CSTAGES - 1;
        if (kn < nk) {
            if (kc >= 1) {   // the stage of chunk kc-1 is free once its MMAs are done
                const bool w = mbar_wait(smem_u32(&mbar[(kc - 1) % CSTAGES]), ((kc - 1) / CSTAGES) & 1);
                if (!__syncthreads_and(w)) { ok = false; break; }
            }
            load(kn, kn % CSTAGES);
            loaded = kn + 1;
        }
        asm volatile("cp.async.commit_group;\n" ::: "memory");
        asm volatile("cp.async.wait_group %0;\n" ::"n"(CSTAGES - 1) : "memory");   // chunk kc's weights
        const bool landed = mbar_wait(smem_u32(&full[s]), (kc / CSTAGES) & 1);      // chunk kc's boxes
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        if (!__syncthreads_and(landed)) { ok = false; break; }
        if (tid == 0) {
            tc_fence_after();
            const unsigned sa = base + s * STAGE, sb = sa + A_BYTES;
            const uint64_t db = sw128_desc(sb);
#pragma unroll
            for (int j = 0; j < GK / 16; j++) {
                const int u = (j * 16) / WC;                        // the box of this K step
                const unsigned off = (unsigned)((j * 16) % WC) * 2;  // bytes into its rows
                const uint64_t da = swk_desc<WC>(sa + u * SUB_BYTES + off);
                const unsigned acc = (kc > 0 || j > 0) ? 1u : 0u;
                asm volatile(
                    "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
                    "l"(da), "l"(db + (uint64_t)(2 * j)), "r"(idesc), "r"(acc));
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                             smem_u32(&mbar[s]))
                         : "memory");
        }
        issued = kc + 1;
    }
    asm volatile("cp.async.wait_all;\n" ::: "memory");
    if (ok && nk > 0) ok = mbar_wait(smem_u32(&mbar[(nk - 1) % CSTAGES]), ((nk - 1) / CSTAGES) & 1);
    ok = __syncthreads_and(ok) != 0;
    if (!ok) {   // leaving early: committed MMAs and issued box copies finish (bounded) before TMEM / smem go
        if (issued > 0) mbar_wait(smem_u32(&mbar[(issued - 1) % CSTAGES]), ((issued - 1) / CSTAGES) & 1);
        if (tid == 0)
            for (int c = loaded - CSTAGES < issued ? issued : loaded - CSTAGES; c < loaded; c++)
                mbar_wait(smem_u32(&full[c % CSTAGES]), (c / CSTAGES) & 1);
        __syncthreads();
    }
    tc_fence_after();

    if (ok) {   // epilogue as k_conv_tc
        const int q = warp & 3, h = warp >> 2;
        const int row = m0 + q * 32 + lane;
        const int half = BN / 2;
        for (int c0 = h * half; c0 < (h + 1) * half; c0 += 8) {
            unsigned r[8];
            const unsigned taddr = tmem + ((unsigned)(q * 32) << 16) + (unsigned)c0;
            asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];\n"
                         : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
                           "=r"(r[7])
                         : "r"(taddr));
            asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
            if (row < M && c0 < N) {
                float v[8];
#pragma unroll
                for (int j = 0; j < 8; j++) {
                    v[j] = (nk > 0 ? __uint_as_float(r[j]) : 0.0f) + (bias ? bias[c0 + j] : 0.0f);
                    if (flags & XBG_NN_RELU) v[j] = fmaxf(v[j], 0.0f);
                }
                if (flags & XBG_NN_OUT_BF16) {
                    __align__(16) __nv_bfloat16 o[8];
#pragma unroll
                    for (int j = 0; j < 8; j++) o[j] = __float2bfloat16(v[j]);
                    *(uint4*)((__nv_bfloat16*)Y + (size_t)row * ldy + c0) = *(const uint4*)o;
                } else {
                    float* d = (float*)Y + (size_t)row * ldy + c0;
                    *(float4*)d = make_float4(v[0], v[1], v[2], v[3]);
                    *(float4*)(d + 4) = make_float4(v[4], v[5], v[6], v[7]);
                }
            }
        }
    } else if (tid == 0) {
        atomicExch(err, XBG_ERR_TIMEOUT);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(TCOLS));
}

// The tensor map of an NHWC bf16 input for k_conv_tma: dims (ldx, W, H, B),
// box (WC, Wt, R, 1) with the WC*2-byte swizzle; false when the shape does
// not tile (W neither a multiple nor a divisor of 128, H not a multiple of R,
// channel counts not multiples of WC, strides not 16-byte multiples).
template <int WC>
bool conv_map(const void* X, int B, int H, int W, int cin, int ldx, CUtensorMap* m) {
    static PFN_cuTensorMapEncodeTiled_v12000 enc = nullptr;
    if (cin % WC || ldx % 8) return false;
    const int Wt = W >= GM ? GM : W;
    if (W >= GM ? (W % GM) : (GM % W)) return false;
    const int R = GM / Wt;
    if (H % R) return false;
    if (!enc) {
        cudaDriverEntryPointQueryResult q;
        void* fn = nullptr;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess || !fn)
            return false;
        enc = (PFN_cuTensorMapEncodeTiled_v12000)fn;
    }
    const cuuint64_t dims[4] = {(cuuint64_t)ldx, (cuuint64_t)W, (cuuint64_t)H, (cuuint64_t)B};
    const cuuint64_t strides[3] = {(cuuint64_t)ldx * 2, (cuuint64_t)W * ldx * 2, (cuuint64_t)H * W * ldx * 2};
    const cuuint32_t box[4] = {(cuuint32_t)WC, (cuuint32_t)Wt, (cuuint32_t)R, 1};
    const cuuint32_t es[4] = {1, 1, 1, 1};
    return enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<void*>(X), dims, strides, box, es,
               CU_TENSOR_MAP_INTERLEAVE_NONE, WC == 32 ? CU_TENSOR_MAP_SWIZZLE_64B : CU_TENSOR_MAP_SWIZZLE_32B,
               CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <int BN, int WC>
int conv_tma_launch(const CUtensorMap& m, const void* Wt, const float* bias, void* Y, int Bn, int H, int W, int cin,
                    int N, int Kp, int ldw, int ldy, int flags, int* err, cudaStream_t st) {
    constexpr int STAGE = GM * GK * 2 + BN * GK * 2;
    const size_t smem = (size_t)CSTAGES * STAGE + 1024;
    static bool attr = false;
    if (!attr) {
        if (cudaFuncSetAttribute(k_conv_tma<BN, WC>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
            cudaSuccess)
            return XBG_ERR_CUDA;
        attr = true;
    }
    const long long M = (long long)Bn * H * W;
    k_conv_tma<BN, WC><<<(unsigned)((M + GM - 1) / GM), 256, smem, st>>>(m, (const __nv_bfloat16*)Wt, bias, Y, Bn,
                                                                          H, W, cin, N, Kp, ldw, ldy, flags, err);
    return cudaGetLastError() == cudaSuccess ? XBG_OK : XBG_ERR_CUDA;
}

// whether xbg_nn_conv3x3 moves its input with box copies (test switch of the
// thread-gathered path, xbg_nn_conv_set_tma)
static int g_conv_tma = 1;

template <int BN>
int conv_launch(const void* X, const void* Wt, const float* bias, void* Y, int Bn, int H, int W, int cin, int ldx,
                int N, int Kp, int ldw, int ldy, int flags, int* err, cudaStream_t st) {
    constexpr int STAGE = GM * GK * 2 + BN * GK * 2;
    const size_t smem = (size_t)CSTAGES * STAGE + 1024;
    static bool attr = false;
    if (!attr) {
        if (cudaFuncSetAttribute(k_conv_tc<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
            return XBG_ERR_CUDA;
        attr = true;
    }
    const long long M = (long long)Bn * H * W;
    if (g_conv_tma && M % GM == 0) {   // box copies of the input when the shape tiles
        CUtensorMap m;
        if (cin % 32 == 0 && conv_map<32>(X, Bn, H, W, cin, ldx, &m))
            return conv_tma_launch<BN, 32>(m, Wt, bias, Y, Bn, H, W, cin, N, Kp, ldw, ldy, flags, err, st);
        if (cin % 32 != 0 && conv_map<16>(X, Bn, H, W, cin, ldx, &m))
            return conv_tma_launch<BN, 16>(m, Wt, bias, Y, Bn, H, W, cin, N, Kp, ldw, ldy, flags, err, st);
    }
    k_conv_tc<BN><<<(unsigned)((M + GM - 1) / GM), 256, smem, st>>>((const __nv_bfloat16*)X,
                                                                     (const __nv_bfloat16*)Wt, bias, Y, Bn, H, W, cin,
                                                                     ldx, N, Kp, ldw, ldy, flags, err);
    return cudaGetLastError() == cudaSuccess ? XBG_OK : XBG_ERR_CUDA;
}


// ------------------------------------------------------------------------
// Weight (and bias) gradient of the 3x3 convolution as an implicit GEMM over
// the pixels:
//
//   D[k][n] = sum over pixels p of col[p][k] dz[p][n],
//   col[p][tap*cin + c] = x[b, y+dy, x+dx, c] (0 outside the image),
//   col[p][9*cin] = 1 (the bias row: D[9*cin][n] = sum_p dz[p][n]).
//
// M = k (128 rows of gw^T per CTA tile), N = n (BN, the layer's padded
// output channels), K = pixels (64 per chunk).  Both operands are indexed
// by pixel rows with the M or N index contiguous in global memory, so both
// are staged "MN-major": a swizzle atom is 8 pixels x W elements (W = 64,
// 32 or 16 with the 128-, 64- or 32-byte swizzle), atoms of one operand
// laid out [MN atom][pixel group] so that a K step of 16 pixels advances
// the descriptor by two atoms.  Each CTA reduces a contiguous range of
// pixel chunks (gridDim.y ranges) into its own slice of `part`; a second
// kernel adds the slices in a fixed order, so the result does not depend
// on scheduling.
__device__ __forceinline__ uint64_t mn_desc(unsigned saddr, unsigned lbo, unsigned sbo, unsigned layout) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);
    d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;   // stride between atoms along M/N
    d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;   // stride between 8-pixel groups
    d |= (uint64_t)1 << 46;
    d |= (uint64_t)layout << 61;
    return d;
}

template <int BN>
__global__ void __launch_bounds__(256, 2) k_wgrad_tc(const __nv_bfloat16* __restrict__ X,
                                                     const __nv_bfloat16* __restrict__ Dz, float* __restrict__ part,
                                                     int Bn, int H, int W, int cin, int ldx, int ldz, int ldp,
                                                     int bias_row, int* err) {
    constexpr int A_BYTES = GM * GK * 2;   // 128 k x 64 pixels
    constexpr int B_BYTES = BN * GK * 2;   // BN n x 64 pixels
    constexpr int STAGE = A_BYTES + B_BYTES;
    constexpr int TCOLS = BN <= 32 ? 32 : (BN <= 64 ? 64 : (BN <= 128 ? 128 : 256));
    // B operand atom: WB channels (a multiple of 16 dividing BN)
    constexpr int WB = (BN % 64 == 0) ? 64 : ((BN % 32 == 0) ? 32 : 16);
    constexpr int AB = WB * 2 * 8;                       // bytes of one atom
    constexpr unsigned BMSK = WB == 64 ? 7u : (WB == 32 ? 3u : 1u);
    constexpr unsigned BLAYOUT = WB == 64 ? 2u : (WB == 32 ? 4u : 6u);
    constexpr int BCH = BN / 8;                          // 16-B pieces per pixel row of B
    extern __shared__ unsigned char smem_raw[];
    __shared__ __align__(8) unsigned long long mbar[CSTAGES];
    __shared__ unsigned tmem_slot;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int P = Bn * H * W;
    const int Kc = 9 * cin;
    const int m0 = blockIdx.x * GM;
    const int nch = (P + GK - 1) / GK;
    const int per = (nch + gridDim.y - 1) / gridDim.y;
    const int kb = blockIdx.y * per, ke = min(nch, kb + per);
    const int nk = max(0, ke - kb);
    const unsigned base = (smem_u32(smem_raw) + 1023u) & ~1023u;
    unsigned char* gbase = smem_raw + (base - smem_u32(smem_raw));
    // this thread's A piece: 8 consecutive k of one tap (fixed for the CTA)
    const int c8 = tid & 15;
    const int kcol = m0 + c8 * 8;
    const int tap = kcol / cin, ch = kcol - tap * cin;
    const int tdy = tap / 3 - 1, tdx = tap % 3 - 1;
    const bool kval = kcol < Kc;
    const bool kbias = bias_row && kcol == Kc;
    const unsigned a_off = (unsigned)((c8 >> 3) * 8192);   // MN atom of the piece
    // image coordinates of this thread's four A rows (pixels p0 + (tid>>4) + 16u
    // of the next chunk to load), advanced by 64 pixels per loaded chunk
    int ax[4], ay[4], ab[4];
#pragma unroll
    for (int u = 0; u < 4; u++) {
        const int p = kb * GK + (tid >> 4) + 16 * u;
        const int t = p / W;
        ax[u] = p - t * W;
        ab[u] = t / H;
        ay[u] = t - ab[u] * H;
    }

    auto load = [&](int kc, int s) {   // called for kc = 0, 1, 2, ... in order
        const unsigned sa = base + s * STAGE, sb = sa + A_BYTES;
        const int p0 = (kb + kc) * GK;
#pragma unroll
        for (int u = 0; u < 4; u++) {   // A: 64 pixels x 16 pieces
            const int r = (tid >> 4) + 16 * u;
            const int p = p0 + r;
            const unsigned dst = sa + a_off + (unsigned)((r >> 3) * 1024 + (r & 7) * 128 + (((c8 & 7) ^ (r & 7)) << 4));
            const int sy = ay[u] + tdy, sx = ax[u] + tdx;
            if (kval && p < P && sy >= 0 && sy < H && sx >= 0 && sx < W)
                cp16(dst, X + ((size_t)(ab[u] * H + sy) * W + sx) * ldx + ch);
            else
                *(uint4*)(gbase + (dst - base)) = make_uint4((kbias && p < P) ? 0x3F80u : 0u, 0u, 0u, 0u);
            ax[u] += GK;
            while (ax[u] >= W) {
                ax[u] -= W;
                if (++ay[u] == H) { ay[u] = 0; ++ab[u]; }
            }
        }
        for (int q = tid; q < GK * BCH; q += 256) {   // B: 64 pixels x BCH pieces
            const int r = q / BCH, c = q - r * BCH;
            const int p = p0 + r;
            const unsigned lin = (unsigned)((c / (WB / 8)) * 8 * AB + (r >> 3) * AB + (r & 7) * (2 * WB) +
                                            (c % (WB / 8)) * 16);
            const unsigned dst = sb + (lin ^ (((lin >> 7) & BMSK) << 4));
            if (p < P) cp16(dst, Dz + (size_t)p * ldz + c * 8);
            else *(uint4*)(gbase + (dst - base)) = make_uint4(0, 0, 0, 0);
        }
    };

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(&tmem_slot)),
                     "r"(TCOLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
    }
    if (tid == 0) {
        for (int s = 0; s < CSTAGES; s++) mbar_init(smem_u32(&mbar[s]), 1);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const unsigned tmem = tmem_slot;
    const uint32_t idesc = idesc_bf16(GM, BN) | (1u << 15) | (1u << 16);   // A and B MN-major
    bool ok = true;
    int issued = 0;
    for (int kc = 0; kc < CSTAGES - 1; kc++) {
        if (kc < nk) load(kc, kc);
        asm volatile("cp.async.commit_group;\n" ::: "memory");
    }
    for (int kc = 0; kc < nk; kc++) {
        const int s = kc % CSTAGES;
        const int kn = kc + CSTAGES - 1;
        if (kn < nk) {
            if (kc >= 1) {
                const bool w = mbar_wait(smem_u32(&mbar[(kc - 1) % CSTAGES]), ((kc - 1) / CSTAGES) & 1);
                if (!__syncthreads_and(w)) { ok = false; break; }
            }
            load(kn, kn % CSTAGES);
        }
        asm volatile("cp.async.commit_group;\n" ::: "memory");
        asm volatile("cp.async.wait_group %0;\n" ::"n"(CSTAGES - 1) : "memory");
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            tc_fence_after();
            const unsigned sa = base + s * STAGE, sb = sa + A_BYTES;
#pragma unroll
            for (int j = 0; j < GK / 16; j++) {   // 16 pixels = two 8-pixel groups per step
                const uint64_t da = mn_desc(sa + j * 2048, 8192, 1024, 2);
                const uint64_t db = mn_desc(sb + j * 2 * AB, 8 * AB, AB, BLAYOUT);
                const unsigned acc = (kc > 0 || j > 0) ? 1u : 0u;
                asm volatile(
                    "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
                    "l"(da), "l"(db), "r"(idesc), "r"(acc));
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                             smem_u32(&mbar[s]))
                         : "memory");
        }
        issued = kc + 1;
    }
    asm volatile("cp.async.wait_all;\n" ::: "memory");
    if (ok && nk > 0) ok = mbar_wait(smem_u32(&mbar[(nk - 1) % CSTAGES]), ((nk - 1) / CSTAGES) & 1);
    ok = __syncthreads_and(ok) != 0;
    if (!ok && issued > 0)
        mbar_wait(smem_u32(&mbar[(issued - 1) % CSTAGES]), ((issued - 1) / CSTAGES) & 1);
    tc_fence_after();

    if (ok) {   // warp w -> TMEM lanes (k rows) 32*(w%4).., column half w/4; part[split][n][k]
        const int q = warp & 3, h = warp >> 2;
        const int row = m0 + q * 32 + lane;
        const int half = BN / 2;
        float* dst = part + (size_t)blockIdx.y * BN * ldp;
        const int kmax = Kc + (bias_row ? 1 : 0);
        for (int c0 = h * half; c0 < (h + 1) * half; c0 += 8) {
            unsigned r[8];
            const unsigned taddr = tmem + ((unsigned)(q * 32) << 16) + (unsigned)c0;
            asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];\n"
                         : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
                           "=r"(r[7])
                         : "r"(taddr));
            asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
            if (row < kmax) {
#pragma unroll
                for (int j = 0; j < 8; j++) dst[(size_t)(c0 + j) * ldp + row] = nk > 0 ? __uint_as_float(r[j]) : 0.0f;
            }
        }
    } else if (tid == 0) {
        atomicExch(err, XBG_ERR_TIMEOUT);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(TCOLS));
}

// gw[n][k] (+)= sum over s of part[s][n][k] (k < Kc), gb[n] (+)= the bias
// row.  Block (32, 8) covers 128 consecutive k of one n, four per thread
// (16-B loads); thread row j adds slices j, j+8, j+16, ... into two
// accumulators (alternating), then thread row 0 adds the sixteen partial sums
// in a fixed order -- the same order whatever the scheduling.
__global__ void k_wgrad_reduce(const float* __restrict__ part, float* __restrict__ gw, float* __restrict__ gb, int N,
                               int Kc, int ldp, int ldw, int ks, int accumulate) {
    __shared__ float4 red[8][33];
    const int kmax = Kc + (gb ? 1 : 0);
    const int k = (blockIdx.x * 32 + threadIdx.x) * 4, n = blockIdx.y, j = threadIdx.y;
    float4 s0 = make_float4(0.f, 0.f, 0.f, 0.f), s1 = s0;
    if (k < kmax) {
        const float* src = part + (size_t)n * ldp + k;
        const size_t step = (size_t)N * ldp;
        int i = j;
        for (; i + 8 < ks; i += 16) {
            const float4 a = *(const float4*)(src + (size_t)i * step);
            const float4 b = *(const float4*)(src + (size_t)(i + 8) * step);
            s0.x += a.x; s0.y += a.y; s0.z += a.z; s0.w += a.w;
            s1.x += b.x; s1.y += b.y; s1.z += b.z; s1.w += b.w;
        }
        if (i < ks) {
            const float4 a = *(const float4*)(src + (size_t)i * step);
            s0.x += a.x; s0.y += a.y; s0.z += a.z; s0.w += a.w;
        }
    }
    red[j][threadIdx.x] = make_float4(s0.x + s1.x, s0.y + s1.y, s0.z + s1.z, s0.w + s1.w);
    __syncthreads();
    if (j != 0 || k >= kmax) return;
    float4 t = red[0][threadIdx.x];
#pragma unroll
    for (int r = 1; r < 8; r++) {
        const float4 v = red[r][threadIdx.x];
        t.x += v.x; t.y += v.y; t.z += v.z; t.w += v.w;
    }
    const float tv[4] = {t.x, t.y, t.z, t.w};
#pragma unroll
    for (int e = 0; e < 4; e++) {
        const int kk = k + e;
        if (kk >= kmax) break;
        float* d = kk < Kc ? gw + (size_t)n * ldw + kk : gb + n;
        *d = accumulate ? *d + tv[e] : tv[e];
    }
}

template <int BN>
int wgrad_launch(const void* X, const void* Dz, float* gw, float* gb, float* work, int Bn, int H, int W, int cin,
                 int ldx, int ldz, int ldw, int ksplit, int accumulate, int* err, cudaStream_t st) {
    constexpr int STAGE = GM * GK * 2 + BN * GK * 2;
    const size_t smem = (size_t)CSTAGES * STAGE + 1024;
    static bool attr = false;
    if (!attr) {
        if (cudaFuncSetAttribute(k_wgrad_tc<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
            cudaSuccess)
            return XBG_ERR_CUDA;
        attr = true;
    }
    const int Kc = 9 * cin;
    const int ldp = Kc + 8;
    const int bias_row = gb ? 1 : 0;
    dim3 grid((unsigned)((Kc + bias_row + GM - 1) / GM), (unsigned)ksplit);
    k_wgrad_tc<BN><<<grid, 256, smem, st>>>((const __nv_bfloat16*)X, (const __nv_bfloat16*)Dz, work, Bn, H, W, cin,
                                            ldx, ldz, ldp, bias_row, err);
    if (cudaGetLastError() != cudaSuccess) return XBG_ERR_CUDA;
    k_wgrad_reduce<<<dim3((unsigned)((Kc + bias_row + 127) / 128), BN), dim3(32, 8), 0, st>>>(work, gw, gb, BN, Kc,
                                                                                             ldp, ldw, ksplit,
                                                                                             accumulate);
    return cudaGetLastError() == cudaSuccess ? XBG_OK : XBG_ERR_CUDA;
}

}  // namespace nn
}  // namespace xbg

extern "C" int xbg_nn_conv_set_tma(int on) {
    xbg::nn::g_conv_tma = on ? 1 : 0;
    return XBG_OK;
}

extern "C" int xbg_nn_conv3x3(const void* X, const void* Wt, const float* bias, void* Y, int B, int H, int W,
                              int cin, int ldx, int N, int Kp, int ldw, int ldy, int flags, int* err, void* stream) {
    using namespace xbg::nn;
    const long long M = (long long)B * H * W;
    if (!X || !Wt || !Y || !err || B < 1 || H < 1 || W < 1 || M > 0x7fffffffLL || cin < 8 || (cin % 8) ||
        (ldx % 8) || ldx < cin || Kp < 9 * cin || (Kp % GK) || ldw < Kp || (ldw % 8) || N < 16 || N > 256 ||
        (N % 16) || ldy < N || (ldy % 8) || (flags & XBG_NN_ATOMIC))
        return XBG_ERR_ARG;
    if (((uintptr_t)X | (uintptr_t)Wt | (uintptr_t)Y) & 15) return XBG_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    switch (N) {
        case 16: return conv_launch<16>(X, Wt, bias, Y, B, H, W, cin, ldx, N, Kp, ldw, ldy, flags, err, st);
        case 32: return conv_launch<32>(X, Wt, bias, Y, B, H, W, cin, ldx, N, Kp, ldw, ldy, flags, err, st);
        case 48: return conv_launch<48>(X, Wt, bias, Y, B, H, W, cin, ldx, N, Kp, ldw, ldy, flags, err, st);
        case 64: return conv_launch<64>(X, Wt, bias, Y, B, H, W, cin, ldx, N, Kp, ldw, ldy, flags, err, st);
        case 96: return conv_launch<96>(X, Wt, bias, Y, B, H, W, cin, ldx, N, Kp, ldw, ldy, flags, err, st);
        case 128: return conv_launch<128>(X, Wt, bias, Y, B, H, W, cin, ldx, N, Kp, ldw, ldy, flags, err, st);
        case 192: return conv_launch<192>(X, Wt, bias, Y, B, H, W, cin, ldx, N, Kp, ldw, ldy, flags, err, st);
        case 256: return conv_launch<256>(X, Wt, bias, Y, B, H, W, cin, ldx, N, Kp, ldw, ldy, flags, err, st);
    }
    return XBG_ERR_ARG;
}

extern "C" int xbg_nn_gemm(const void* A, const void* B, const float* bias, void* C, int M, int N, int K, int lda,
                           int ldb, int ldc, int flags, int ksplit, int* err, void* stream) {
    using namespace xbg::nn;
    if (!A || !B || !C || !err || M < 1 || K < GK || (K % GK) || N < 16 || N > 256 || (N % 16) || (lda % 8) ||
        (ldb % 8) || lda < K || ldb < K || ldc < N || ksplit < 1 || ksplit > 65535)
        return XBG_ERR_ARG;
    if ((flags & XBG_NN_ATOMIC) && (flags & XBG_NN_OUT_BF16)) return XBG_ERR_ARG;
    if (ksplit > 1 && !(flags & XBG_NN_ATOMIC)) return XBG_ERR_ARG;
    if (((uintptr_t)A | (uintptr_t)B) & 15) return XBG_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    switch (N) {
        case 16: return gemm_launch<16>(A, B, bias, C, M, N, K, lda, ldb, ldc, flags, ksplit, err, st);
        case 32: return gemm_launch<32>(A, B, bias, C, M, N, K, lda, ldb, ldc, flags, ksplit, err, st);
        case 48: return gemm_launch<48>(A, B, bias, C, M, N, K, lda, ldb, ldc, flags, ksplit, err, st);
        case 64: return gemm_launch<64>(A, B, bias, C, M, N, K, lda, ldb, ldc, flags, ksplit, err, st);
        case 96: return gemm_launch<96>(A, B, bias, C, M, N, K, lda, ldb, ldc, flags, ksplit, err, st);
        case 128: return gemm_launch<128>(A, B, bias, C, M, N, K, lda, ldb, ldc, flags, ksplit, err, st);
        case 192: return gemm_launch<192>(A, B, bias, C, M, N, K, lda, ldb, ldc, flags, ksplit, err, st);
        case 256: return gemm_launch<256>(A, B, bias, C, M, N, K, lda, ldb, ldc, flags, ksplit, err, st);
    }
    return XBG_ERR_ARG;
}

extern "C" long long xbg_nn_conv3x3_wgrad_work(int cin, int N, int ksplit) {
    return (long long)ksplit * N * (9LL * cin + 8);
}

extern "C" int xbg_nn_conv3x3_wgrad(const void* X, const void* Dz, float* gw, float* gb, float* work, int B, int H,
                                    int W, int cin, int ldx, int N, int ldz, int ldw, int ksplit, int accumulate,
                                    int* err, void* stream) {
    using namespace xbg::nn;
    const long long P = (long long)B * H * W;
    if (!X || !Dz || !gw || !work || !err || B < 1 || H < 1 || W < 1 || P > 0x7fffffffLL || cin < 8 || (cin % 8) ||
        (ldx % 8) || ldx < cin || (ldz % 8) || ldz < N || ldw < 9 * cin || ksplit < 1 || ksplit > 65535 ||
        9LL * cin + 8 > 0x7fffffffLL / 256)
        return XBG_ERR_ARG;
    if (((uintptr_t)X | (uintptr_t)Dz | (uintptr_t)work) & 15) return XBG_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    switch (N) {
        case 16: return wgrad_launch<16>(X, Dz, gw, gb, work, B, H, W, cin, ldx, ldz, ldw, ksplit, accumulate, err, st);
        case 32: return wgrad_launch<32>(X, Dz, gw, gb, work, B, H, W, cin, ldx, ldz, ldw, ksplit, accumulate, err, st);
        case 48: return wgrad_launch<48>(X, Dz, gw, gb, work, B, H, W, cin, ldx, ldz, ldw, ksplit, accumulate, err, st);
        case 64: return wgrad_launch<64>(X, Dz, gw, gb, work, B, H, W, cin, ldx, ldz, ldw, ksplit, accumulate, err, st);
        case 96: return wgrad_launch<96>(X, Dz, gw, gb, work, B, H, W, cin, ldx, ldz, ldw, ksplit, accumulate, err, st);
        case 128: return wgrad_launch<128>(X, Dz, gw, gb, work, B, H, W, cin, ldx, ldz, ldw, ksplit, accumulate, err, st);
        case 192: return wgrad_launch<192>(X, Dz, gw, gb, work, B, H, W, cin, ldx, ldz, ldw, ksplit, accumulate, err, st);
        case 256: return wgrad_launch<256>(X, Dz, gw, gb, work, B, H, W, cin, ldx, ldz, ldw, ksplit, accumulate, err, st);
    }
    return XBG_ERR_ARG;
}
