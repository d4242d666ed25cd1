// noalloc.cu -- xbg_flow_dt_noalloc: the flow time-step limit of the step
// (the FLOWDT minimum that k_step_begin reduces) for caller-owned device
// arrays, without allocating any device memory.
//
// The result is the FLOWDT part of xbg_compute_dt bit for bit (same maximum
// depth, same single square root, same rounding).
//
// Who needs it: a host code that couples this model into its own solver and
// has handed the whole device to its own pool allocator (an ocean or
// atmosphere coupler, an ML framework's caching allocator) may not allocate
// behind that allocator's back; and cudaMalloc/cudaFree synchronise the
// whole device, which stalls every other stream of a caller that overlaps
// work.  Such a caller owns hh and the output; the only memory beyond those
// that the reduction needs (one minimum per block and a completion counter)
// lives in the file-scope array below, reserved once when the library loads.
//
// Limits and sharing:
//   * scratch: XBG_NOALLOC_SCRATCH_BYTES (256 B counter line + one 8-byte
//     minimum for each of at most XBG_NOALLOC_MAX_BLOCKS blocks), held by
//     every GPU that loads the library until the process exits;
//   * at most XBG_NOALLOC_MAX_CELLS cells (32-bit cell index with room for
//     the grid stride); larger grids are rejected with XBG_ERR_ARG before
//     any device work;
//   * every call on a device shares the one array: calls that can overlap on
//     the GPU (two streams, two threads) race and must be ordered by the
//     caller.  The completion counter is cleared on the caller's stream
//     before each launch; the per-block minima need no clearing (each launch
//     writes every slot it later reads).
//   * the first call on a device (the current device) looks up the device
//     address of the array (cudaGetSymbolAddress) and keeps it for the life
//     of the process; make that first call before any stream capture on that
//     device.  After cudaDeviceReset the kept address is stale: reload the
//     library (a new process) before calling it again.
#include <mutex>

#include "xbg_common.cuh"
#include "../../include/xbg.h"

namespace xbg {

// The scratch array.  In host code this name is only a stand-in for the
// symbol: the device address comes from cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char na_scratch[XBG_NOALLOC_SCRATCH_BYTES];

namespace {

constexpr int NA_THREADS = 256;
constexpr int NA_MAX_DEVICES = 64;
static_assert(XBG_NOALLOC_SCRATCH_BYTES >= 256 + 8 * XBG_NOALLOC_MAX_BLOCKS, "scratch too small");

std::mutex na_mu;

// max of two block depth maxima, where -1 marks a block that saw a
// non-finite depth and must win
template <class R>
__device__ __forceinline__ R na_max(R a, R b) { return (a < (R)0 || b < (R)0) ? (R)-1 : DM<R>::fmax(a, b); }
void* na_addr[NA_MAX_DEVICES] = {};

// Same limit and reduction as k_step_begin's FLOWDT part (Wave_kernel.cu:161,
// Wave_gpu.cu:620-640): cfl*dx/sqrt(g*hh) falls as hh grows, so the minimum
// over cells is the limit at the deepest cell; each block reduces the maximum
// depth, the last block to finish reduces the block maxima and takes one
// square root.  No block waits on another.  Writes 0.5 * the minimum (the dt
// candidate of the step), 3.0e38 * 0.5 when no depth is positive, and NaN
// when any depth is NaN or infinite.
template <class R>
__global__ void __launch_bounds__(NA_THREADS) k_flow_dt_noalloc(const R* __restrict__ hh, int n, R cfl, R dx,
                                                                 unsigned char* scratch, R* out) {
    unsigned* counter = reinterpret_cast<unsigned*>(scratch);
    R* part = reinterpret_cast<R*>(scratch + 256);
    __shared__ R red[NA_THREADS / 32];
    __shared__ int last;
    int tid = threadIdx.x;
    R hmax = (R)0, probe = (R)0;   // probe: sum of hh * 0, zero only if every depth is finite
    for (int i = blockIdx.x * NA_THREADS + tid; i < n; i += gridDim.x * NA_THREADS) {
        const R h = ld(hh + i);
        hmax = DM<R>::fmax(hmax, h);
        probe = probe + h * (R)0;
    }
    if (!(probe == (R)0)) hmax = (R)-1;   // marks the block; carried by the max below as NaN
    for (int o = 16; o > 0; o >>= 1) hmax = na_max(hmax, __shfl_xor_sync(0xffffffffu, hmax, o));
    if ((tid & 31) == 0) red[tid >> 5] = hmax;
    __syncthreads();
    if (tid == 0) {
        R b = red[0];
        for (int w = 1; w < NA_THREADS / 32; w++) b = na_max(b, red[w]);
        part[blockIdx.x] = b;
        __threadfence();
        last = (atomicAdd(counter, 1u) == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    R hm = (R)0;
    for (int j = tid; j < (int)gridDim.x; j += NA_THREADS) hm = na_max(hm, ((volatile R*)part)[j]);
    for (int o = 16; o > 0; o >>= 1) hm = na_max(hm, __shfl_xor_sync(0xffffffffu, hm, o));
    __syncthreads();
    if ((tid & 31) == 0) red[tid >> 5] = hm;
    __syncthreads();
    if (tid == 0) {
        for (int w = 0; w < NA_THREADS / 32; w++) hm = na_max(hm, red[w]);
        R mf = (R)3.0e38f;
        if (hm < (R)0) mf = (R)NAN;   // a block saw a non-finite depth
        else if (hm > (R)0) mf = cfl * dx / (DM<R>::sqrt((R)9.81f * hm));
        *out = (R)0.5 * mf;
        *counter = 0;
    }
}

// Device address of na_scratch on the current device, looked up once.
int na_scratch_addr(unsigned char** out) {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess) return XBG_ERR_CUDA;
    if (dev < 0 || dev >= NA_MAX_DEVICES) return XBG_ERR_ARG;
    std::lock_guard<std::mutex> lk(na_mu);
    if (!na_addr[dev]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, na_scratch) != cudaSuccess || !p) return XBG_ERR_CUDA;
        na_addr[dev] = p;
    }
    *out = static_cast<unsigned char*>(na_addr[dev]);
    return XBG_OK;
}

template <class R>
int flow_dt_noalloc(const void* hh, int n, double dx, double cfl, void* dt_out, cudaStream_t st) {
    unsigned char* scratch = nullptr;
    int rc = na_scratch_addr(&scratch);
    if (rc) return rc;
    int nb = (n + NA_THREADS - 1) / NA_THREADS;
    if (nb > XBG_NOALLOC_MAX_BLOCKS) nb = XBG_NOALLOC_MAX_BLOCKS;
    if (cudaMemsetAsync(scratch, 0, sizeof(unsigned), st) != cudaSuccess) return XBG_ERR_CUDA;
    k_flow_dt_noalloc<R><<<nb, NA_THREADS, 0, st>>>(static_cast<const R*>(hh), n, (R)cfl, (R)dx, scratch,
                                                     static_cast<R*>(dt_out));
    return cudaGetLastError() == cudaSuccess ? XBG_OK : XBG_ERR_CUDA;
}

}  // namespace
}  // namespace xbg

extern "C" int xbg_flow_dt_noalloc(int precision, const void* hh, int nx, int ny, double dx, double cfl,
                                   void* dt_out, void* stream) {
    if (precision != XBG_FP32 && precision != XBG_FP64) return XBG_ERR_ARG;
    if (nx < 1 || ny < 1 || (long long)nx * ny > XBG_NOALLOC_MAX_CELLS) return XBG_ERR_ARG;
    if (!hh || !dt_out || !(dx > 0.0) || !(cfl > 0.0)) return XBG_ERR_ARG;
    int n = nx * ny;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    return precision == XBG_FP32 ? xbg::flow_dt_noalloc<float>(hh, n, dx, cfl, dt_out, st)
                                 : xbg::flow_dt_noalloc<double>(hh, n, dx, cfl, dt_out, st);
}
