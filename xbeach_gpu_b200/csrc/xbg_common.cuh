// xbg_common.cuh -- device-side state, constants and helpers shared by the
// wave, flow, sediment and time-step kernels.
//
// Layout in HBM (one handle): structure of arrays, cell i = ix + iy*nx, every
// 2-D field a separate cudaMalloc'd array of nx*ny elements (float or double),
// directional fields as ntheta planes of nx*ny (the reference's layout,
// Wave_kernel.cu:264).  ee and rr have two planes sets each; the step whose
// device clock flips `par` reads set par^1 and writes set par, so a captured
// CUDA graph can replay any number of steps without pointer swaps.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#define XBG_PI 3.14159265          /* the reference's `pi` macro (double) */
#define XBG_MAX_THETA 32

namespace xbg {

// --------------------------------------------------------------- math
// Float functions for float, double functions for double: the FP64 build is
// the same kernels instantiated on double.
template <class R> struct DM;
template <> struct DM<float> {
    static __device__ __forceinline__ float sqrt(float x) { return sqrtf(x); }
    static __device__ __forceinline__ float sinh(float x) { return sinhf(x); }
    static __device__ __forceinline__ float tanh(float x) { return tanhf(x); }
    static __device__ __forceinline__ float pow(float x, float y) { return powf(x, y); }
    // x^(1/3) and x^(2/3) with the exponents the reference writes as float
    // literals (1.0f/3.0f, 0.66666666667f).  FP32: cbrtf (within 1e-7
    // relative of powf with those exponents); FP64: pow with the same
    // float-valued exponents, as the reference evaluates them.
    static __device__ __forceinline__ float pow13(float x) { return cbrtf(x); }
    static __device__ __forceinline__ float pow23(float x) { float c = cbrtf(x); return c * c; }
    static __device__ __forceinline__ float exp(float x) { return expf(x); }
    static __device__ __forceinline__ float log(float x) { return logf(x); }
    static __device__ __forceinline__ float log10(float x) { return log10f(x); }
    static __device__ __forceinline__ float cos(float x) { return cosf(x); }
    static __device__ __forceinline__ float sin(float x) { return sinf(x); }
    static __device__ __forceinline__ void sincos(float x, float* s, float* c) { sincosf(x, s, c); }
    static __device__ __forceinline__ float fabs(float x) { return fabsf(x); }
    static __device__ __forceinline__ float fmin(float a, float b) { return fminf(a, b); }
    static __device__ __forceinline__ float fmax(float a, float b) { return fmaxf(a, b); }
    static __device__ __forceinline__ float fma(float a, float b, float c) { return fmaf(a, b, c); }
    // a product the compiler may not fuse into an fma (fixes the rounding of
    // a*b +- c*d expressions whatever the surrounding code)
    static __device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
    static __device__ __forceinline__ float atan(float x) { return atanf(x); }
};
template <> struct DM<double> {
    static __device__ __forceinline__ double sqrt(double x) { return ::sqrt(x); }
    static __device__ __forceinline__ double sinh(double x) { return ::sinh(x); }
    static __device__ __forceinline__ double tanh(double x) { return ::tanh(x); }
    static __device__ __forceinline__ double pow(double x, double y) { return ::pow(x, y); }
    static __device__ __forceinline__ double pow13(double x) { return ::pow(x, (double)(1.0f / 3.0f)); }
    static __device__ __forceinline__ double pow23(double x) { return ::pow(x, (double)0.66666666667f); }
    static __device__ __forceinline__ double exp(double x) { return ::exp(x); }
    static __device__ __forceinline__ double log(double x) { return ::log(x); }
    static __device__ __forceinline__ double log10(double x) { return ::log10(x); }
    static __device__ __forceinline__ double cos(double x) { return ::cos(x); }
    static __device__ __forceinline__ double sin(double x) { return ::sin(x); }
    static __device__ __forceinline__ void sincos(double x, double* s, double* c) { ::sincos(x, s, c); }
    static __device__ __forceinline__ double fabs(double x) { return ::fabs(x); }
    static __device__ __forceinline__ double fmin(double a, double b) { return ::fmin(a, b); }
    static __device__ __forceinline__ double fmax(double a, double b) { return ::fmax(a, b); }
    static __device__ __forceinline__ double fma(double a, double b, double c) { return ::fma(a, b, c); }
    static __device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
    static __device__ __forceinline__ double atan(double x) { return ::atan(x); }
};

// min/max as the reference's CPU wave code defines them (wave_CPU.cpp:10-16);
// the flow and sediment kernels use CUDA's fminf/fmaxf semantics (DM::fmin).
template <class T> __device__ __forceinline__ T cmax(T a, T b) { return (a < b) ? b : a; }
template <class T> __device__ __forceinline__ T cmin(T a, T b) { return !(b < a) ? a : b; }

// Clamped neighbours (Wave_kernel.cu:23-77, Flow_CPU.cpp:16-70).
__device__ __forceinline__ int mm(int i) { return i <= 0 ? 0 : i - 1; }
__device__ __forceinline__ int pp(int i, int n) { return i >= n - 1 ? n - 1 : i + 1; }
__device__ __forceinline__ int mm2(int i) { return i <= 1 ? 0 : i - 2; }
__device__ __forceinline__ int pp2(int i, int n) { return i >= n - 2 ? n - 1 : i + 2; }

template <class T> __device__ __forceinline__ T ld(const T* p) { return __ldg(p); }

// --------------------------------------------------------------- state
enum Fld {
    ZB = 0, ZS, HH, UU, VV, HU, HV, HUM, HVM, QX, QY, UEU, VEV, VMAGEU, VMAGEV, VU, UV,
    UUOLD, VVOLD, ZSOLD, DZSDT, H, E, D, DR, ROL, WK, CC_, CG, FX, FY, URMS, UST, THM,
    CFM, FWM, CSED, CEQSG, STDEP, DZB, ROLTHICK, KTURB, HMEAN, UUMEAN, VVMEAN, HHMEAN,
    ZSMEAN, CMEAN, ZSMAX, NF2D
};
// Per-step temporaries (never read across steps).
enum Tmp {
    T_UU = 0, T_VV, T_ZS, T_NUH, T_SXX, T_SXY, T_SYY, T_CEQBG, T_TSG, T_UA, T_FACERO,
    T_ERO, T_DEPO, T_ZB, T_STDEP, T_HH, T_QX, T_QY, NTMP
};

template <class R>
struct Dev {
    int nx, ny, nt, C;
    R* f[NF2D];
    R* tmp[NTMP];
    int* wetu;
    int* wetv;
    R* umeanbnd;          // ny
    R* ee[2];             // two plane sets of nt*C
    R* rr[2];
    R* St;                // interpolated offshore boundary, nt*ny
    R* stfile[2];         // boundary chunk slots: nrec*nt*ny
    R* qfile[2];          // nrec*4*ny
    R* part_flow;         // per-block FLOWDT minima
    R* part_wave;         // per-block WAVEDT minima
    R* zsold[2];          // zsold ping-pong, selected by the clock's par
    unsigned* counter;    // last-block-done counter of the dt reduction
    struct Clock* clk;
};

// Device clock and boundary cursors: the globals of mainloopGPU, wavebnd and
// flowbnd (Wave_gpu.cu:26-241, Wavestep.cu:512-753) kept in device memory.
struct Clock {
    double totaltime, dt, nextoutputtime;
    float wdt;                 // previous dt, a float in the reference (Wave_gpu.cu:78)
    int par;                   // which ee/rr plane set holds the current state
    int halt;                  // 1: the rest of this step is skipped
    int forced;                // 1: the wave sub-step comes from a forcing (surrogate), the wave kernels skip
    int flags;                 // XBG_FLAG_*
    int status;                // XBG_OK or XBG_ERR_*
    int do_sed;                // sedimentstep runs this step
    long long nstep, nstep_total;
    // wave boundary
    int cur_slot;
    int slot_valid[2];
    int slot_nrec[2];
    double slot_t0[2], slot_tend[2], slot_Trep[2];
    int WAVstep;               // wavebndtype 1 record cursor
    int nwbndstep;
    double timenext_w, timesincelast_w;
    double Trep;               // float in the reference, stored rounded
    double sigm;               // 2 pi / Trep rounded to the element type
    // sea level and wind
    int SLstep, WNDstep, nsl, nwnd;
    double zsbndi, zsbndn, windu, windv;
    int n_wave_parts;          // number of valid WAVEDT partials (0 = none)
};
static_assert(offsetof(Clock, forced) == offsetof(Clock, halt) + sizeof(int) && offsetof(Clock, halt) % 8 == 0,
              "halt and forced form one aligned 8-byte word (read together by wave_off)");
static_assert(sizeof(Clock) == 240, "XBG_CLOCK_BYTES in xbg.h is the clock's size");
#define XBG_MAX_SERIES 4096
struct Series {
    double slt[XBG_MAX_SERIES], sla[XBG_MAX_SERIES], slb[XBG_MAX_SERIES];
    double wt[XBG_MAX_SERIES], wa[XBG_MAX_SERIES], wb[XBG_MAX_SERIES];
    double wavet[XBG_MAX_SERIES];   // wavebndtype 1 record times
};

// Constants of one handle, passed by value to every kernel.
template <class R>
struct Konst {
    int nx, ny, nt;
    int swave, flow, roller, breakmodel, usesmago, wavebndtype, means;
    R dx, eps, g, rho, cfl, dtheta, gammax, gammaa, alpha, nexp, beta, wci, hwci;
    R nuh, nuhfac, fc, Cd, D50, D90, rhosed, wws, drydzmax, wetdzmax, maxslpchg, por,
        morfac, sus, facsk, facas, cfsand, cfreef, fwsand, fwreef;
    R twopi, aphi, bphi;
    // run constants of Sbvr / Rvr (Sediment_kernel.cu:167-326, 477-509),
    // evaluated once on the host: drho*g, Ass, the Ucr prefactor
    // (0.19 D50^0.1 or 8.5 D50^0.6), Rvr's alpha and beta; and 1/dx
    R sed_drho, sed_drhog, sed_Ass, sed_ucr, rvr_alpha, rvr_beta, rdx;
    double endtime, outputtimestep, sedstart, dtbc, eps_d;
    int sedtrans;
    R cxsth[XBG_MAX_THETA], sxnth[XBG_MAX_THETA], theta[XBG_MAX_THETA];
};

// Tensor maps of the wave rows pass (TMA variant): ee and rr of both plane
// sets, box loads of one bin's plane tile and box stores of all bins of a
// block's cells.  Passed to the kernel as a __grid_constant__ parameter.
struct WaveMaps {
    CUtensorMap ld_e[2], ld_r[2], st_e[2], st_r[2];
};

// Per-kernel timing of a non-graph step (xbg_profile_step): an event after
// every launch on the handle's stream.
struct Prof {
    cudaEvent_t ev[65];
    const char* name[64];
    int n = 0;
    cudaStream_t st = nullptr;
    void mark(const char* nm) {
        if (n < 64) { name[n] = nm; cudaEventRecord(ev[n + 1], st); n++; }
    }
};
#define PMARK(pf, nm) do { if (pf) (pf)->mark(nm); } while (0)

// ---------------------------------------------------------------- tiles
// Asynchronous 4/8-byte global -> shared copies (cp.async) and their groups.
template <int BYTES>
__device__ __forceinline__ void cp_async(void* smem, const void* gmem) {
    unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(sa), "l"(gmem), "n"(BYTES));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;\n" ::); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::); }

// A block's cell tile (32 x 8 cells, 256 threads) with a halo of H cells,
// filled with the grid clamped at its edges: the tile element next to a cell
// is the neighbour the reference reads through mm()/pp()/mm2()/pp2().
template <int H>
struct TileG {
    static constexpr int X = 32, Y = 8, TX = X + 2 * H, TY = Y + 2 * H, N = TX * TY;
};

// Copy NF fields over the tile (cp.async), then wait and synchronise the
// block.  Fields 0 and 1 (the water level and the bed in every staged pass,
// read together by the wet tests) are interleaved, t[2 e + f], so a tile
// cell's pair is one 8-byte (16-byte) shared-memory load; field f >= 2 is
// the plane t[f * N + e].
template <class R, int H, int NF>
__device__ __forceinline__ void tile_load(R* t, const R* const (&src)[NF], int bx0, int by0, int nx, int ny) {
    using G = TileG<H>;
    const int tid = threadIdx.x + threadIdx.y * G::X;
    for (int e = tid; e < G::N; e += G::X * G::Y) {
        int gx = min(max(bx0 - H + e % G::TX, 0), nx - 1), gy = min(max(by0 - H + e / G::TX, 0), ny - 1);
        size_t g = (size_t)gx + (size_t)gy * nx;
        cp_async<sizeof(R)>(t + 2 * e, src[0] + g);
        cp_async<sizeof(R)>(t + 2 * e + 1, src[1] + g);
#pragma unroll
        for (int f = 2; f < NF; f++) cp_async<sizeof(R)>(t + f * G::N + e, src[f] + g);
    }
    cp_async_commit();
    cp_async_wait_all();
    __syncthreads();
}
template <class R> struct Pair2 { R a, b; };
template <class R> struct alignas(2 * sizeof(R)) Pair2A { R a, b; };

// Tile index of the cell that tile position (kx, ky) stands for (the grid
// clamped), and that cell's grid coordinates.
template <int H>
__device__ __forceinline__ int tile_centre(int kx, int ky, int bx0, int by0, int nx, int ny, int& gx, int& gy) {
    using G = TileG<H>;
    int vx = bx0 - H + kx, vy = by0 - H + ky;
    gx = min(max(vx, 0), nx - 1);
    gy = min(max(vy, 0), ny - 1);
    return (ky + gy - vy) * G::TX + (kx + gx - vx);
}

// Field access around one cell: a(f, dx, dy) = field f at
// (clamp(ix + dx), clamp(iy + dy)), from the shared-memory tile ...
// zz(dx, dy): fields 0 and 1 there together.
template <class R, int H>
struct TileAt {
    const R* t;
    int k;
    __device__ __forceinline__ R operator()(int f, int dx, int dy) const {
        const int p = k + dx + dy * TileG<H>::TX;
        return f < 2 ? t[2 * p + f] : t[f * TileG<H>::N + p];
    }
    __device__ __forceinline__ Pair2<R> zz(int dx, int dy) const {
        const Pair2A<R> v = reinterpret_cast<const Pair2A<R>*>(t)[k + dx + dy * TileG<H>::TX];
        return Pair2<R>{v.a, v.b};
    }
};
// ... or from global memory.
template <class R, int NF>
struct GlobalAt {
    const R* p[NF];
    int ix, iy, nx, ny;
    __device__ __forceinline__ R operator()(int f, int dx, int dy) const {
        int x = min(max(ix + dx, 0), nx - 1), y = min(max(iy + dy, 0), ny - 1);
        return __ldg(p[f] + x + (size_t)y * nx);
    }
    __device__ __forceinline__ Pair2<R> zz(int dx, int dy) const {
        return Pair2<R>{(*this)(0, dx, dy), (*this)(1, dx, dy)};
    }
};
// Minima of fields 0 and 1 (level and bed) over the window x in [x0, x1],
// y in [y0, y1] around a cell, one pair load per window cell.
template <class R, class A>
__device__ __forceinline__ Pair2<R> zz_min(const A& a, int x0, int x1, int y0, int y1) {
    Pair2<R> m = a.zz(x0, y0);
    for (int dy = y0; dy <= y1; dy++)
        for (int dx = (dy == y0 ? x0 + 1 : x0); dx <= x1; dx++) {
            const Pair2<R> v = a.zz(dx, dy);
            m.a = DM<R>::fmin(m.a, v.a);
            m.b = DM<R>::fmin(m.b, v.b);
        }
    return m;
}

// Row segments: a thread takes V consecutive cells of one row (V = 4 in
// FP32, 2 in FP64) with one 16-byte load per field and row, and a warp one
// row of 32 V cells; the cells left and right of a thread's segment come from
// the adjacent lanes (the first and last lane of a warp load theirs), and
// mm()/pp() clamping at the grid's edges gives the segment's own end cell.
// Needs nx a multiple of V (row starts 16-byte aligned).  Every lane of a
// warp takes part in the shuffles, including lanes past the row's end.
template <class R> struct SegVec;
template <> struct SegVec<float> { using T = float4; using I = int4; static constexpr int V = 4; };
template <> struct SegVec<double> { using T = double2; using I = int2; static constexpr int V = 2; };
template <class R>
struct Seg {
    using VT = typename SegVec<R>::T;
    using VI = typename SegVec<R>::I;
    static constexpr int V = SegVec<R>::V;
    union U { VT v; R a[V]; };
    union W { VI v; int a[V]; };
    int nx, x0, lane;
    bool act;   // the segment lies in the row
    __device__ __forceinline__ Seg(int nx_, int bx) : nx(nx_), lane((int)threadIdx.x) {
        x0 = (bx * (int)blockDim.x + lane) * V;
        act = x0 < nx;
    }
    __device__ __forceinline__ size_t at(int y) const { return (size_t)y * nx + x0; }
    __device__ __forceinline__ U row(const R* f, int y) const {
        U u;
        if (act) u.v = __ldg(reinterpret_cast<const VT*>(f + at(y)));
        else
            for (int k = 0; k < V; k++) u.a[k] = (R)0;
        return u;
    }
    // the cell left of the segment (mm: the segment's first cell at column 0)
    __device__ __forceinline__ R left(const U& u, const R* f, int y) const {
        R w = __shfl_up_sync(0xffffffffu, u.a[V - 1], 1);
        if (lane == 0 && act && x0 > 0) w = __ldg(f + at(y) - 1);
        return x0 > 0 ? w : u.a[0];
    }
    // the cell right of the segment (pp: the segment's last cell at column nx-1)
    __device__ __forceinline__ R right(const U& u, const R* f, int y) const {
        R w = __shfl_down_sync(0xffffffffu, u.a[0], 1);
        if (lane == 31 && act && x0 + V < nx) w = __ldg(f + at(y) + V);
        return x0 + V < nx ? w : u.a[V - 1];
    }
    __device__ __forceinline__ void put(R* f, int y, const U& u) const { *reinterpret_cast<VT*>(f + at(y)) = u.v; }
    __device__ __forceinline__ void put(int* f, int y, const W& w) const { *reinterpret_cast<VI*>(f + at(y)) = w.v; }
};

// ---------------------------------------------------------------- batches
// A batch advances many scenarios (each with its own grid, parameters, clock
// and dt) with one launch per kernel of the step.  Each kernel is a body
// b_NAME(S, K, bx, by) over one block-sized tile; the single-domain kernel
// k_NAME runs it at (blockIdx.x, blockIdx.y), the batched kernel kb_NAME runs
// it for each (scenario, tile) work item of its list, persistent blocks
// taking contiguous runs of items.

// Per-scenario extras that single-domain kernels get as launch arguments.
struct BatchAux {
    const Series* ser;
    int nflow;          // blocks of the dt reduction
    int nwave;          // WAVEDT partials
    int ubnd_threads;   // logical thread count of the ubnd block
    int scen;           // the scenario's index in the batch
};

template <class R>
struct BatchTab {
    const Dev<R>* S;
    const Konst<R>* K;
    const BatchAux* A;
};

// Work-item lists, one per tile shape: (scenario, bx | by << 16)
enum BatchShape {
    BS_TILE,    // 32 x 8 tiles over nx x ny
    BS_WROWS,   // 32 x 8 tiles over nx x rows 1..ny-2 (wave pass)
    BS_LIN,     // 256-cell runs of the C cells
    BS_ONE,     // one block per scenario
    BS_BND,     // 256-value runs of the ny*ntheta boundary values
    BS_DT,      // the blocks of the dt reduction
    BS_WIDE,    // 64 x 4 tiles over nx x ny (the pointwise passes' other shape)
    BS_N
};
struct BatchLaunch {
    const int2* items[BS_N];
    int n[BS_N];
    int grid[BS_N];
};

template <class R, class F>
__device__ __forceinline__ void batch_items(const BatchTab<R>& T, const int2* items, int n, F&& f) {
    constexpr int WD = (int)(sizeof(Dev<R>) / 4), WK = (int)(sizeof(Konst<R>) / 4), WA = (int)(sizeof(BatchAux) / 4);
    __shared__ __align__(16) unsigned sbuf[WD + WK + WA];
    const Dev<R>& sS = *reinterpret_cast<const Dev<R>*>(sbuf);
    const Konst<R>& sK = *reinterpret_cast<const Konst<R>*>(sbuf + WD);
    const BatchAux& sA = *reinterpret_cast<const BatchAux*>(sbuf + WD + WK);
    const int tid = threadIdx.x + blockDim.x * threadIdx.y;
    const int nth = blockDim.x * blockDim.y;
    const int per = (n + gridDim.x - 1) / gridDim.x;
    const int lo = blockIdx.x * per, hi = min(n, lo + per);
    int cur = -1;
    for (int it = lo; it < hi; it++) {
        const int2 w = items[it];
        if (w.x != cur) {   // stage the scenario's state and constants
            __syncthreads();
            const unsigned* gS = reinterpret_cast<const unsigned*>(T.S + w.x);
            const unsigned* gK = reinterpret_cast<const unsigned*>(T.K + w.x);
            const unsigned* gA = reinterpret_cast<const unsigned*>(T.A + w.x);
            for (int k = tid; k < WD + WK + WA; k += nth)
                sbuf[k] = k < WD ? gS[k] : (k < WD + WK ? gK[k - WD] : gA[k - WD - WK]);
            __syncthreads();
            cur = w.x;
        }
        f(sS, sK, sA, w.y & 0xffff, w.y >> 16);
        __syncthreads();
    }
}

// Single-domain and batched kernels of a 256-thread body b_NAME(S, K, bx, by).
#define XBG_BATCH_KERNEL(NAME)                                                                         \
    template <class R>                                                                                 \
    __global__ void __launch_bounds__(256) kb_##NAME(BatchTab<R> T, const int2* items, int n) {        \
        batch_items<R>(T, items, n, [&](const Dev<R>& S, const Konst<R>& K, const BatchAux&, int bx,   \
                                        int by) { b_##NAME<R>(S, K, bx, by); });                       \
    }
#define XBG_KERNELS(NAME)                                                                              \
    template <class R>                                                                                 \
    __global__ void __launch_bounds__(256) k_##NAME(Dev<R> S, Konst<R> K) {                            \
        b_##NAME<R>(S, K, blockIdx.x, blockIdx.y);                                                     \
    }                                                                                                  \
    XBG_BATCH_KERNEL(NAME)

// Early exit of a kernel in a step that the device clock has halted.  The
// flow passes, the second sediment pass and the dispersion pass read the
// flag with their first loads and test it just before their first store,
// behind a compiler barrier, so the flag's round trip overlaps the field
// loads instead of preceding them (a halted step computes and discards;
// nothing is stored).  Where a kernel timed faster testing it up front
// (the other sediment passes, the wave force pass) it does that.
__device__ __forceinline__ void loads_before_here() { asm volatile("" ::: "memory"); }
__device__ __forceinline__ bool halted(const Clock* c) {
    return *((volatile const int*)&c->halt) != 0;
}
// ... and of the wave solver's kernels while a forcing replaces them (halt
// and forced in one load).
__device__ __forceinline__ bool wave_off(const Clock* c) {
    return *((volatile const unsigned long long*)&c->halt) != 0ull;
}

}  // namespace xbg
