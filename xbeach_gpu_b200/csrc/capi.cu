// capi.cu -- host side of the C ABI declared in include/xbg.h.
//
// One handle owns every device buffer of one model, one CUDA stream and one
// captured CUDA graph of a whole coupled step.  Nothing here synchronises the
// stream except the calls that return host data (get_field, get_time, mass)
// and the boundary upload, which must know which chunk slot is in use.
#include <cuda_runtime.h>
#include <cmath>
#include <cstring>
#include <cstdio>
#include <map>
#include <vector>
#include <algorithm>
#include "xbg_common.cuh"
#include "../../include/xbg.h"
#include "../../include/xbg_io.h"

// the wave rows variant a new handle or batch starts with (1: TMA tiles, one
// cell per thread; 2: TMA tiles, two cells per thread)
#ifndef XBG_WAVE_VARIANT_DEFAULT
#define XBG_WAVE_VARIANT_DEFAULT 1
#endif
// the flow variant they start with (0: momentum steps in two passes, 1: one;
// the two passes are the faster at 2048 x 1024, the fused one on smaller grids)
#ifndef XBG_FLOW_VARIANT_DEFAULT
#define XBG_FLOW_VARIANT_DEFAULT 0
#endif

namespace xbg {
template <class R> int launch_wave(const Dev<R>&, const Konst<R>&, cudaStream_t, Prof*, cudaEvent_t, const WaveMaps*, int,
                                   bool);
template <class R> int wave_maps_make(const Dev<R>&, const Konst<R>&, WaveMaps*);
template <class R> int wave_parts(const Konst<R>&);
template <class R> int wave_prepare(const Konst<R>&);
template <class R> int launch_flow(const Dev<R>&, const Konst<R>&, cudaStream_t, Prof*, bool, bool, bool);
template <class R> int launch_sed(const Dev<R>&, const Konst<R>&, cudaStream_t, Prof*, bool, bool);
template <class R> int step_begin_blocks(const Konst<R>&);
template <class R> int launch_step_begin(const Dev<R>&, const Konst<R>&, const Series*, int, cudaStream_t, Prof*);
template <class R> int launch_ubnd(const Dev<R>&, const Konst<R>&, const Series*, cudaStream_t, Prof*);
template <class R> int launch_wavebnd(const Dev<R>&, const Konst<R>&, const Series*, cudaStream_t, Prof*, int);
template <class R> int launch_means(const Dev<R>&, const Konst<R>&, cudaStream_t, Prof*);
template <class R> int launch_step_begin_batch(const BatchTab<R>&, const BatchLaunch&, cudaStream_t, Prof*);
template <class R> int launch_wavebnd_batch(const BatchTab<R>&, const BatchLaunch&, cudaStream_t, Prof*);
template <class R> int launch_ubnd_batch(const BatchTab<R>&, const BatchLaunch&, cudaStream_t, Prof*);
template <class R> int launch_means_batch(const BatchTab<R>&, const BatchLaunch&, cudaStream_t, Prof*);
template <class R> int launch_wave_batch(const BatchTab<R>&, const BatchLaunch&, int, int, int, cudaStream_t, Prof*,
                                         cudaEvent_t, const WaveMaps*, int, bool);
template <class R> int launch_flow_batch(const BatchTab<R>&, const BatchLaunch&, cudaStream_t, Prof*, bool, bool);
template <class R> int launch_sed_batch(const BatchTab<R>&, const BatchLaunch&, cudaStream_t, Prof*, bool);
template <class R> int ubnd_threads(const Konst<R>&);
template <class R> void launch_output_done(const Dev<R>&, const Konst<R>&, cudaStream_t);
template <class R> void launch_reset_means(const Dev<R>&, cudaStream_t);
template <class R> void launch_mass(const Dev<R>&, double, double*, cudaStream_t);

template <class R>
__global__ void k_set_slot(Clock* c, int logical, int nrec, double t0, double tend, double Trep) {
    int phys = logical == 0 ? c->cur_slot : (c->cur_slot ^ 1);
    c->slot_valid[phys] = 1;
    c->slot_nrec[phys] = nrec;
    c->slot_t0[phys] = t0;
    c->slot_tend[phys] = tend;
    c->slot_Trep[phys] = Trep;
    if (logical == 1) c->flags &= ~XBG_FLAG_NEED_BOUNDARY;
}
// Wave forcing from outside the wave solver (the surrogate): E, H, D, DR, Fx,
// Fy = f0 + w (f1 - f0) (E, H, D, DR clipped at 0).  With rescale, the wave
// action of every bin in both plane sets (still the state that f0 describes)
// scales by E_new / E0 and the roller energy (both sets and R) by DR_new /
// DR0, so a later plain wave step starts from the state the forcing
// describes.
template <class R>
struct Forcing6 { const R* p[6]; };

template <class R>
__device__ __forceinline__ void set_forcing_cell(const Dev<R>& S, R* ee0, R* ee1, R* rr0, R* rr1,
                                                 const R* const* f0, const R* const* f1, R w, int rescale, int i) {
    R v[6];
#pragma unroll
    for (int c = 0; c < 6; c++) v[c] = f0[c][i] + w * (f1[c][i] - f0[c][i]);
#pragma unroll
    for (int c = 0; c < 4; c++) v[c] = v[c] > (R)0 ? v[c] : (R)0;
    if (rescale) {   // ee, rr still hold the state of f0 (the segment start)
        const R Eo = f0[0][i], DRo = f0[3][i];
        const R re = Eo > (R)1e-12 ? v[0] / Eo : (R)1;
        const R rr = DRo > (R)1e-12 ? v[3] / DRo : (R)1;
        for (int t = 0; t < S.nt; t++) {
            const size_t j = (size_t)i + (size_t)t * S.C;
            ee0[j] *= re; ee1[j] *= re;
            rr0[j] *= rr; rr1[j] *= rr;
        }
        S.f[ROL][i] *= rr;
    }
    S.f[E][i] = v[0]; S.f[H][i] = v[1]; S.f[D][i] = v[2]; S.f[DR][i] = v[3]; S.f[FX][i] = v[4]; S.f[FY][i] = v[5];
}
template <class R>
__global__ void k_set_forcing(Dev<R> S, R* ee0, R* ee1, R* rr0, R* rr1, Forcing6<R> f0, Forcing6<R> f1, R w,
                              int rescale) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= S.C) return;
    set_forcing_cell(S, ee0, ee1, rr0, rr1, f0.p, f1.p, w, rescale, i);
}

// The forcing planes of each scenario of a batch (xbg_batch_set_forcing).
template <class R>
struct ForcingPair { const R* f0[6]; const R* f1[6]; };

// The forcing of every scenario in forced mode, one 256-cell run per item;
// scenarios in plain mode (their wave solver ran this step) are left alone.
template <class R>
__global__ void __launch_bounds__(256) kb_set_forcing(BatchTab<R> T, const ForcingPair<R>* fp, R w, int rescale,
                                                      const int2* items, int n) {
    batch_items<R>(T, items, n, [&](const Dev<R>& S, const Konst<R>&, const BatchAux& A, int bx, int) {
        if (halted(S.clk) || *((volatile const int*)&S.clk->forced) == 0) return;
        const int i = bx * 256 + threadIdx.x;
        if (i >= S.C) return;
        const ForcingPair<R>& f = fp[A.scen];
        set_forcing_cell(S, S.ee[0], S.ee[1], S.rr[0], S.rr[1], f.f0, f.f1, w, rescale, i);
    });
}

// Per scenario sum((pred - field)^2) and sum(field^2) (FP64 accumulators,
// one pair per scenario); scenarios without a prediction are skipped.
template <class R>
struct ErrPair { const R* field; const R* pred; };
template <class R>
__global__ void __launch_bounds__(256) kb_rel_err(BatchTab<R> T, const ErrPair<R>* ep, double* acc,
                                                  const int2* items, int n) {
    batch_items<R>(T, items, n, [&](const Dev<R>& S, const Konst<R>&, const BatchAux& A, int bx, int) {
        const ErrPair<R> e = ep[A.scen];
        if (!e.pred) return;
        const int i = bx * 256 + threadIdx.x;
        double d2 = 0.0, f2 = 0.0;
        if (i < S.C) {
            const double f = (double)e.field[i], d = (double)e.pred[i] - f;
            d2 = d * d;
            f2 = f * f;
        }
        for (int o = 16; o > 0; o >>= 1) {
            d2 += __shfl_xor_sync(0xffffffffu, d2, o);
            f2 += __shfl_xor_sync(0xffffffffu, f2, o);
        }
        if ((threadIdx.x & 31) == 0) {
            atomicAdd(acc + 2 * A.scen, d2);
            atomicAdd(acc + 2 * A.scen + 1, f2);
        }
    });
}

// wave mode of one clock: forced (1) or plain (0); fallback also marks it
__global__ void k_set_wave_mode(Clock* c, int forced, int fallback) {
    c->forced = forced;
    if (fallback) c->flags |= XBG_FLAG_FALLBACK;
}

// Copy every scenario's device clock of a batch into one array.
template <class R>
__global__ void k_gather_clocks(const Dev<R>* S, int n, Clock* out) {
    int s = blockIdx.x;
    if (s >= n) return;
    const unsigned* src = reinterpret_cast<const unsigned*>(S[s].clk);
    unsigned* dst = reinterpret_cast<unsigned*>(out + s);
    for (int k = threadIdx.x; k < (int)(sizeof(Clock) / 4); k += blockDim.x) dst[k] = src[k];
}

}  // namespace xbg

using namespace xbg;

// ------------------------------------------------------------------ params
extern "C" void xbg_params_default(xbg_params* p) {   // XBeachGPU.h:62-154
    std::memset(p, 0, sizeof(*p));
    p->swave = 1; p->flow = 1; p->sedtrans = 0; p->morphology = 0;
    p->g = 9.81; p->rho = 1025.0; p->eps = 0.01;
    p->cf = 0.01; p->cfsand = 0.0; p->cfreef = 0.0;
    p->nuh = 1.0; p->nuhfac = 1.0; p->usesmago = 1; p->smag = 0.3;
    p->lat = 0.0; p->fc = 0.0; p->Cd = 0.002; p->wci = 0.0; p->hwci = 0.1;
    p->breakmodel = 1; p->gammaa = 0.6; p->n = 8.0; p->alpha = 1.0; p->gammax = 2.0; p->beta = 0.15;
    p->fw = 0.001; p->fwsand = 0.0; p->fwreef = 0.0;
    p->roller = 1;
    p->thetamin = -90 * 3.14159265 / 180; p->thetamax = 90 * 3.14159265 / 180;
    p->dtheta = 0.0; p->ntheta = 0;
    p->D50 = 0.00038; p->D90 = 0.00053; p->rhosed = 2650.0; p->wws = 0.0509;
    p->drydzmax = 1.0; p->wetdzmax = 0.3; p->maxslpchg = 0.01; p->por = 0.4; p->morfac = 1.0;
    p->sus = 1.0; p->bed = 1.0; p->facsk = 0.2; p->facas = 0.2;
    p->wavebndtype = 2;
    p->CFL = 0.7; p->sedstart = 3600.0; p->outputtimestep = 0.0; p->endtime = 0.0;
    p->dtbc = 1.0; p->rtlength = 3600.0;
    p->means = 1;
}

// checkparamsanity (read_input.cpp:1227-1443, the step-path rules), the
// theta bins of waveinitGPU (Wavestep.cu:33-45) and the Coriolis parameter
// (Wave_gpu.cu:2060-2064).
extern "C" int xbg_params_sanity(xbg_params* p, double endbnd) {
    const double tiny = 0.0000001;
    if (p->nx <= 0 || p->ny <= 0 || p->dx < tiny) return XBG_ERR_ARG;
    if (std::fabs(p->endtime - 0.0) <= tiny) p->endtime = 1.0 / tiny;
    p->endtime = std::min(p->endtime, endbnd);
    if (p->swave == 0) { p->ntheta = 1; p->dtheta = p->thetamax - p->thetamin; }
    if (std::fabs(p->outputtimestep) <= tiny) p->outputtimestep = p->endtime;
    if (std::fabs(p->cfsand) < tiny) { if (p->cf < tiny) p->cf = tiny; p->cfsand = p->cf; }
    if (std::fabs(p->cfreef) < tiny) p->cfreef = p->cfsand;
    if (std::fabs(p->fwsand) < tiny) { if (p->fw < tiny) p->fw = tiny; p->fwsand = p->fw; }
    if (std::fabs(p->fwreef) < tiny) p->fwreef = p->fwsand;
    if (p->usesmago == 1) p->nuh = p->smag;
    if (p->swave == 1) {
        if (p->dtheta > 0.0) p->ntheta = (int)std::round((p->thetamax - p->thetamin) / p->dtheta);
        else { if (p->ntheta == 0) p->ntheta = 1; p->dtheta = (p->thetamax - p->thetamin) / p->ntheta; }
    }
    double wearth = 3.14159265 * (1.0 / 24.0) / 1800.0;
    p->fc = 2.0 * wearth * std::sin(p->lat);
    return XBG_OK;
}

extern "C" const char* xbg_status_string(int s) {
    switch (s) {
        case XBG_OK: return "ok";
        case XBG_ERR_ARG: return "bad argument";
        case XBG_ERR_CUDA: return "CUDA error";
        case XBG_ERR_NAN: return "model crashed: dt is 0, inf or NaN";
        case XBG_ERR_DT: return "initial time step below 1e-8";
        case XBG_ERR_TIMEOUT: return "device wait timed out";
        case XBG_ERR_STATE: return "call out of order";
        case XBG_ERR_NOMEM: return "out of device memory";
        case XBG_ERR_BOUNDARY: return "ran past the uploaded wave boundary";
        case XBG_ERR_IO: return "file could not be opened or written";
        case XBG_ERR_FORMAT: return "input file format error";
    }
    return "unknown status";
}

// ------------------------------------------------------------------ handle
struct xbg_handle {
    virtual ~xbg_handle() {}
    xbg_params P;
    int precision = XBG_FP32;
    int64_t launches = 0;
    cudaStream_t ext = nullptr;   // a batch's stream that also works on this state
    bool batch_owned = false;      // destroyed with its batch only
    virtual int init_state(const void* zb, double zs0, double zs1) = 0;
    virtual int field_count(int f, size_t* n) = 0;
    virtual int set_field(int f, const void* p, size_t n) = 0;
    virtual int get_field(int f, void* p, size_t n) = 0;
    virtual int device_ptr(int f, void** p, size_t* n) = 0;
    virtual int set_wave_boundary(int slot, const double* St, const double* q, int nrec,
                                  const double* times, double t0, double tend, double Trep) = 0;
    virtual int set_series(int which, const double* t, const double* a, const double* b, int n) = 0;
    virtual int piece(int which) = 0;
    virtual int step(int nsteps) = 0;
    virtual int get_time(double* t, double* dt, int64_t* n, int* flags) = 0;
    virtual int get_time_async(void* dst) = 0;
    virtual int state_bytes(size_t* n) = 0;
    virtual int save_state(void* dst, size_t n) = 0;
    virtual int load_state(const void* src, size_t n) = 0;
    virtual int clock_decode(const void* src, double* t, double* dt, int64_t* n, int* flags) = 0;
    virtual int set_time(double t, double dt, double wdt) = 0;
    virtual int output_done() = 0;
    virtual int reset_means() = 0;
    virtual int mass(double* w, double* s, double* b) = 0;
    virtual int sync() = 0;
    virtual void* stream() = 0;
    virtual int profile(float* ms, const char** names, int* n) = 0;
    virtual int put_wave_records(int slot, int first, int n, const void* St, const void* q) = 0;
    virtual int set_forcing(const void* const* f0, const void* const* f1, double w, int rescale) = 0;
    virtual int forcing_steps(const void* const* f0, const void* const* f1, int k) = 0;
    virtual int fetch(const int* fields, int n, void* const* dst) = 0;
    virtual int set_variant(int phase, int variant) = 0;
    virtual int get_variant(int phase, int* variant) = 0;
};

struct xbg_batch {
    virtual ~xbg_batch() {}
    int n = 0;
    std::vector<xbg_handle*> h;
    virtual int advance(int nsteps) = 0;
    virtual int status(double* t, double* dt, int64_t* nstep, int* flags, int* st) = 0;
    virtual int sync() = 0;
    virtual void* stream() = 0;
    virtual int profile(float* ms, const char** names, int* n) = 0;
    virtual int set_grid(int shape, int blocks) = 0;
    virtual int64_t launches() = 0;
    virtual int set_variant(int phase, int variant) = 0;
    virtual int get_variant(int phase, int* variant) = 0;
    virtual int set_wave_mode(int s, int mode) = 0;
    virtual int set_forcing(int s, const void* const* f0, const void* const* f1) = 0;
    virtual int forced_segment(int k) = 0;
    virtual int rel_err(int field, const void* const* pred, double* err) = 0;
};

namespace {

#define CK(x) do { cudaError_t e_ = (x); if (e_ != cudaSuccess) { last_err = e_; return e_ == cudaErrorMemoryAllocation ? XBG_ERR_NOMEM : XBG_ERR_CUDA; } } while (0)

template <class R>
struct Handle : public xbg_handle {
    Dev<R> S;
    Konst<R> K;
    Clock* clk = nullptr;
    Series* ser = nullptr;
    R* zsold_buf[2] = {nullptr, nullptr};
    R* ee_buf[2] = {nullptr, nullptr};
    R* rr_buf[2] = {nullptr, nullptr};
    size_t slot_cap = 0;        // elements of St per slot
    std::vector<void*> allocs;
    cudaStream_t st = nullptr;
    cudaStream_t side = nullptr;          // the boundary kernels' branch of the step graph
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    cudaGraphExec_t gexec = nullptr;
    cudaGraph_t graph = nullptr;
    // graph of a forced segment (xbg_forcing_steps) and what it was captured for
    cudaGraphExec_t seg_exec = nullptr;
    cudaGraph_t seg_graph = nullptr;
    const void* seg_key[13] = {};
    int seg_launches = 0;
    int per_step_launches = 0;
    int nwave = 0;
    cudaError_t last_err = cudaSuccess;
    double* mass_buf = nullptr;
    // wave rows pass: TMA tiles with one cell per thread (variant 1) or two
    // (variant 2), when its maps could be made and wave-current interaction
    // is off, or thread-copied tiles (variant 0)
    WaveMaps maps;
    bool maps_ok = false;
    int wave_variant = XBG_WAVE_VARIANT_DEFAULT;
    const WaveMaps* wave_maps() const { return (maps_ok && wave_variant >= 1) ? &maps : nullptr; }
    int wave_cpt() const { return wave_variant == 2 ? 2 : 1; }
    // flow: momentum steps in one pass (variant 1) or two (variant 0)
    int flow_variant = XBG_FLOW_VARIANT_DEFAULT;
    // the pointwise passes in 32 x 8 (variant 0) or 64 x 4 (variant 1) blocks,
    // or (variant 2, the default where nx is a multiple of the segment width)
    // row segments of 16-byte loads where a pass has that form (the first
    // flow and sediment passes; the others take 32 x 8 blocks)
    int tile_variant = 0;
    bool wide() const { return tile_variant == 1; }
    bool vec() const { return tile_variant == 2; }

    template <class T> int alloc(T** p, size_t n) {
        void* q = nullptr;
        if (n == 0) n = 1;
        CK(cudaMalloc(&q, n * sizeof(T)));
        CK(cudaMemsetAsync(q, 0, n * sizeof(T), st));
        allocs.push_back(q);
        *p = (T*)q;
        return XBG_OK;
    }
    // free one allocation made by alloc() before the handle's end
    void release(void* p) {
        auto it = std::find(allocs.begin(), allocs.end(), p);
        if (it != allocs.end()) {
            allocs.erase(it);
            cudaFree(p);
        }
    }

    int setup(const xbg_params* p, int prec) {
        P = *p;
        precision = prec;
        int nx = P.nx, ny = P.ny, nt = P.ntheta;
        if (nx < 4 || ny < 4 || nt < 1 || nt > XBG_MAX_THETA) return XBG_ERR_ARG;
        size_t C = (size_t)nx * ny;
        CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        CK(cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking));
        CK(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&ev_join, cudaEventDisableTiming));
        std::memset(&S, 0, sizeof(S));
        S.nx = nx; S.ny = ny; S.nt = nt; S.C = (int)C;
        int rc;
        for (int f = 0; f < NF2D; f++) if ((rc = alloc(&S.f[f], C))) return rc;
        for (int f = 0; f < NTMP; f++) if ((rc = alloc(&S.tmp[f], C))) return rc;
        if ((rc = alloc(&S.wetu, C)) || (rc = alloc(&S.wetv, C)) || (rc = alloc(&S.umeanbnd, (size_t)ny))) return rc;
        for (int k = 0; k < 2; k++) {
            if ((rc = alloc(&ee_buf[k], C * nt)) || (rc = alloc(&rr_buf[k], C * nt)) || (rc = alloc(&zsold_buf[k], C)))
                return rc;
            S.ee[k] = ee_buf[k]; S.rr[k] = rr_buf[k]; S.zsold[k] = zsold_buf[k];
        }
        if ((rc = alloc(&S.St, (size_t)ny * nt))) return rc;
        // K
        std::memset(&K, 0, sizeof(K));
        K.nx = nx; K.ny = ny; K.nt = nt;
        K.swave = P.swave; K.flow = P.flow; K.roller = P.roller; K.breakmodel = P.breakmodel;
        K.usesmago = P.usesmago; K.wavebndtype = P.wavebndtype; K.means = P.means;
        K.dx = (R)P.dx; K.eps = (R)P.eps; K.g = (R)P.g; K.rho = (R)P.rho; K.cfl = (R)P.CFL;
        K.dtheta = (R)P.dtheta; K.gammax = (R)P.gammax; K.gammaa = (R)P.gammaa; K.alpha = (R)P.alpha;
        K.nexp = (R)P.n; K.beta = (R)P.beta; K.wci = (R)P.wci; K.hwci = (R)P.hwci;
        K.nuh = (R)P.nuh; K.nuhfac = (R)P.nuhfac; K.fc = (R)P.fc; K.Cd = (R)P.Cd;
        K.D50 = (R)P.D50; K.D90 = (R)P.D90; K.rhosed = (R)P.rhosed; K.wws = (R)P.wws;
        K.drydzmax = (R)P.drydzmax; K.wetdzmax = (R)P.wetdzmax; K.maxslpchg = (R)P.maxslpchg;
        K.por = (R)P.por; K.morfac = (R)P.morfac; K.sus = (R)P.sus; K.facsk = (R)P.facsk;
        K.facas = (R)P.facas; K.cfsand = (R)P.cfsand; K.cfreef = (R)P.cfreef;
        K.fwsand = (R)P.fwsand; K.fwreef = (R)P.fwreef;
        R phi = (R)((1.0f + (R)std::sqrt((R)5.0f)) / 2);
        K.aphi = 1 / (phi + 1); K.bphi = phi / (phi + 1);
        K.twopi = 8 * (R)std::atan((R)1.0f);
        {
            R drho = (K.rhosed - K.rho) / K.rho;
            R dester = (R)std::pow(drho * K.g, (R)(1.0f / 3.0f)) / (R)0.0001f * K.D50;
            K.sed_drho = drho;
            K.sed_drhog = drho * K.g;
            K.sed_Ass = (R)0.012f * K.D50 * (R)std::pow(dester, (R)-0.6f) / (R)std::pow(drho * K.g * K.D50, (R)1.2f);
            K.sed_ucr = K.D50 <= (R)0.0005f ? (R)0.19f * (R)std::pow(K.D50, (R)0.1f)
                                             : (R)8.50f * (R)std::pow(K.D50, (R)0.6f);
            K.rvr_alpha = (R)-1.0f * (R)std::log10((R)std::exp((R)1.0f)) / (R)0.3539f;
            K.rvr_beta = (R)std::exp((R)-0.6065f / (R)0.3539f);
            K.rdx = (R)1 / K.dx;
        }
        K.endtime = P.endtime; K.outputtimestep = P.outputtimestep; K.sedstart = P.sedstart;
        K.dtbc = P.dtbc; K.eps_d = P.eps; K.sedtrans = P.sedtrans;
        for (int i = 0; i < nt; i++) {   // Wavestep.cu:79-86
            K.theta[i] = (R)(i * (P.dtheta) + P.thetamin + 0.5f * P.dtheta);
            K.cxsth[i] = (R)std::cos(K.theta[i]);
            K.sxnth[i] = (R)std::sin(K.theta[i]);
        }
        if (wave_prepare(K)) return XBG_ERR_CUDA;
        maps_ok = K.wci == (R)0 && wave_maps_make(S, K, &maps) == 0;
        // the row-segment passes where the rows split into whole segments
        tile_variant = K.nx % (sizeof(R) == 4 ? 4 : 2) == 0 ? 2 : 0;
        // reductions and clock
        int nflow = step_begin_blocks(K);
        nwave = wave_parts(K);
        if ((rc = alloc(&S.part_flow, (size_t)2 * nflow)) || (rc = alloc(&S.part_wave, (size_t)nwave)) ||
            (rc = alloc(&S.counter, 1)) || (rc = alloc(&clk, 1)) || (rc = alloc(&ser, 1)) ||
            (rc = alloc(&mass_buf, 3)))
            return rc;
        S.clk = clk;
        std::vector<R> big((size_t)nwave, (R)3.0e38f);
        CK(cudaMemcpyAsync(S.part_wave, big.data(), nwave * sizeof(R), cudaMemcpyHostToDevice, st));
        Clock c;
        std::memset(&c, 0, sizeof(c));
        c.nextoutputtime = P.outputtimestep;   // Wave_gpu.cu:2959
        c.WAVstep = 1; c.SLstep = 1; c.WNDstep = 1;
        c.n_wave_parts = nwave;
        CK(cudaMemcpyAsync(clk, &c, sizeof(c), cudaMemcpyHostToDevice, st));
        CK(cudaStreamSynchronize(st));
        return XBG_OK;
    }

    ~Handle() override {
        if (st) cudaStreamSynchronize(st);
        if (gexec) cudaGraphExecDestroy(gexec);
        if (graph) cudaGraphDestroy(graph);
        if (seg_exec) cudaGraphExecDestroy(seg_exec);
        if (seg_graph) cudaGraphDestroy(seg_graph);
        for (void* p : allocs) cudaFree(p);
        if (ev_fork) cudaEventDestroy(ev_fork);
        if (ev_join) cudaEventDestroy(ev_join);
        if (side) cudaStreamDestroy(side);
        if (st) cudaStreamDestroy(st);
    }

    int host_cur_slot = 0;
    int host_par = 0;           // plane set current as of the last clock read
    bool clock_stale = true;    // a step that may flip the set was enqueued since
    int read_clock(Clock& c) {
        if (ext) CK(cudaStreamSynchronize(ext));
        CK(cudaStreamSynchronize(st));
        CK(cudaMemcpy(&c, clk, sizeof(c), cudaMemcpyDeviceToHost));
        host_cur_slot = c.cur_slot;
        host_par = c.par;
        clock_stale = false;
        return XBG_OK;
    }

    // output fields to host memory, stream-ordered; synchronises only when the
    // current plane set of ee/rr/zsold is not known on the host
    int fetch(const int* fields, int n, void* const* dst) override {
        if (n < 0 || (n > 0 && (!fields || !dst))) return XBG_ERR_ARG;
        if (clock_stale || batch_owned) {
            Clock c;
            int rc = read_clock(c);
            if (rc) return rc;
        }
        for (int k = 0; k < n; k++) {
            const int f = fields[k];
            if (!dst[k]) return XBG_ERR_ARG;
            if (f == XBG_F_WETU || f == XBG_F_WETV) {
                CK(cudaMemcpyAsync(dst[k], f == XBG_F_WETU ? S.wetu : S.wetv, (size_t)S.C * sizeof(int),
                                   cudaMemcpyDeviceToHost, st));
                continue;
            }
            size_t m;
            R* d = field_ptr(f, &m, host_par);
            if (!d) return XBG_ERR_ARG;
            CK(cudaMemcpyAsync(dst[k], d, m * sizeof(R), cudaMemcpyDeviceToHost, st));
        }
        return XBG_OK;
    }

    R* field_ptr(int f, size_t* n, int par) {
        size_t C = (size_t)S.C;
        *n = C;
        switch (f) {
            case XBG_F_EE: *n = C * K.nt; return ee_buf[par];
            case XBG_F_RR: *n = C * K.nt; return rr_buf[par];
            case XBG_F_ZSOLD: return zsold_buf[par];
            case XBG_F_UMEANBND: *n = K.ny; return S.umeanbnd;
            default: break;
        }
        static const int map[] = {ZB, ZS, HH, UU, VV, HU, HV, HUM, HVM, QX, QY, UEU, VEV, VMAGEU, VMAGEV,
                                  VU, UV, UUOLD, VVOLD, -1, DZSDT, H, E, D, DR, ROL, WK, CC_, CG, FX, FY,
                                  URMS, UST, THM, CFM, FWM, CSED, CEQSG, STDEP, DZB, ROLTHICK, KTURB,
                                  HMEAN, UUMEAN, VVMEAN, HHMEAN, ZSMEAN, CMEAN, ZSMAX};
        if (f < 0 || f >= (int)(sizeof(map) / sizeof(map[0])) || map[f] < 0) return nullptr;
        return S.f[map[f]];
    }

    int field_count(int f, size_t* n) override {
        if (f == XBG_F_WETU || f == XBG_F_WETV) { *n = (size_t)S.C; return XBG_OK; }
        if (!field_ptr(f, n, 0)) return XBG_ERR_ARG;
        return XBG_OK;
    }
    int set_field(int f, const void* p, size_t n) override {
        Clock c;
        int rc = read_clock(c);
        if (rc) return rc;
        if (f == XBG_F_WETU || f == XBG_F_WETV) {
            if (n != (size_t)S.C) return XBG_ERR_ARG;
            CK(cudaMemcpy(f == XBG_F_WETU ? S.wetu : S.wetv, p, n * sizeof(int), cudaMemcpyHostToDevice));
            return XBG_OK;
        }
        size_t m;
        R* d = field_ptr(f, &m, c.par);
        if (!d || m != n) return XBG_ERR_ARG;
        std::vector<R> clipped;
        if (f == XBG_F_EE) {   // wave energy is kept non-negative in memory (the sanity step of the wave pass)
            const R* src = (const R*)p;
            clipped.resize(n);
            for (size_t j = 0; j < n; j++) clipped[j] = src[j] > (R)0 ? src[j] : (R)0;
            p = clipped.data();
        }
        CK(cudaMemcpy(d, p, n * sizeof(R), cudaMemcpyHostToDevice));
        // double-buffered fields: both sets, so a piece-wise step (without
        // compute_dt flipping the set) reads what was set
        R* other = nullptr;
        if (f == XBG_F_ZSOLD) other = zsold_buf[c.par ^ 1];
        if (f == XBG_F_EE) other = ee_buf[c.par ^ 1];
        if (f == XBG_F_RR) other = rr_buf[c.par ^ 1];
        if (other) CK(cudaMemcpy(other, p, n * sizeof(R), cudaMemcpyHostToDevice));
        return XBG_OK;
    }
    int get_field(int f, void* p, size_t n) override {
        Clock c;
        int rc = read_clock(c);
        if (rc) return rc;
        if (f == XBG_F_WETU || f == XBG_F_WETV) {
            if (n != (size_t)S.C) return XBG_ERR_ARG;
            CK(cudaMemcpy(p, f == XBG_F_WETU ? S.wetu : S.wetv, n * sizeof(int), cudaMemcpyDeviceToHost));
            return XBG_OK;
        }
        size_t m;
        R* d = field_ptr(f, &m, c.par);
        if (!d || m != n) return XBG_ERR_ARG;
        CK(cudaMemcpy(p, d, n * sizeof(R), cudaMemcpyDeviceToHost));
        return XBG_OK;
    }
    int device_ptr(int f, void** p, size_t* n) override {
        Clock c;
        int rc = read_clock(c);
        if (rc) return rc;
        if (f == XBG_F_WETU || f == XBG_F_WETV) { *p = f == XBG_F_WETU ? S.wetu : S.wetv; *n = S.C; return XBG_OK; }
        R* d = field_ptr(f, n, c.par);
        if (!d) return XBG_ERR_ARG;
        *p = d;
        return XBG_OK;
    }

    // Reference initial condition, computed on the host as main() does
    // (Wave_gpu.cu:1988-2015, 2040-2052, 2457-2510, 2637-2692).
    int init_state(const void* zbp, double zs0, double zs1) override {
        int nx = K.nx, ny = K.ny;
        size_t C = (size_t)S.C;
        const R* zbin = (const R*)zbp;
        std::vector<R> zb(zbin, zbin + C), zs(C), hh(C), stdep(C, (R)5.0f), cfm(C), fwm(C);
        for (int iy = 0; iy < ny; iy++)
            for (int ix = 0; ix < nx; ix++) {
                size_t i = ix + (size_t)iy * nx;
                double zsbnd = zs0 + (zs1 - zs0) * (iy) / ny;
                R a = (R)zsbnd, b = (R)(-1 * zb[i]);
                zs[i] = (a < b) ? b : a;
                double h = (double)zb[i] + zsbnd;
                hh[i] = (R)((h < P.eps) ? P.eps : h);
            }
        for (size_t i = 0; i < C; i++) {   // updatezom
            if (stdep[i] < (R)0.05f) { cfm[i] = (R)P.cfreef; fwm[i] = (R)P.fwreef; }
            else { cfm[i] = (R)P.cfsand; fwm[i] = (R)P.fwsand; }
        }
        // initial dt: FLOWDT with 0.5*CFL, minimum, times 0.5 (Wave_gpu.cu:2648-2679)
        R cfl = (R)(0.5f * P.CFL);
        double mn = 1e300;
        for (size_t i = 0; i < C; i++) {
            R v = cfl * (R)P.dx / (std::sqrt((R)9.81f * hh[i]));
            mn = std::min(mn, (double)v);
        }
        double dt0 = (double)(R)mn * 0.5;
        if (dt0 < 0.00000001) return XBG_ERR_DT;
        CK(cudaMemcpy(S.f[ZB], zb.data(), C * sizeof(R), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(S.f[ZS], zs.data(), C * sizeof(R), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(S.f[HH], hh.data(), C * sizeof(R), cudaMemcpyHostToDevice));
        for (int f : {HU, HV, HUM, HVM}) CK(cudaMemcpy(S.f[f], hh.data(), C * sizeof(R), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(S.f[STDEP], stdep.data(), C * sizeof(R), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(S.f[CFM], cfm.data(), C * sizeof(R), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(S.f[FWM], fwm.data(), C * sizeof(R), cudaMemcpyHostToDevice));
        Clock c;
        int rc = read_clock(c);
        if (rc) return rc;
        CK(cudaMemcpy(zsold_buf[c.par], zs.data(), C * sizeof(R), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(zsold_buf[c.par ^ 1], zs.data(), C * sizeof(R), cudaMemcpyHostToDevice));
        c.dt = dt0;
        c.wdt = (float)dt0;
        if (P.swave == 1) {
            if (!c.slot_valid[c.cur_slot]) return XBG_ERR_STATE;
            R Trep = (R)c.slot_Trep[c.cur_slot];
            c.Trep = (double)Trep;
            c.sigm = (double)(R)(2.0f * 3.14159265 / (double)Trep);
            // ee column 0 from the first record (Wavestep.cu:355-375)
            std::vector<R> col((size_t)ny * K.nt);
            CK(cudaMemcpy(col.data(), S.stfile[c.cur_slot], col.size() * sizeof(R), cudaMemcpyDeviceToHost));
            for (int t = 0; t < K.nt; t++)
                CK(cudaMemcpy2D(ee_buf[c.par] + (size_t)t * C, (size_t)nx * sizeof(R), &col[(size_t)t * ny],
                                sizeof(R), sizeof(R), ny, cudaMemcpyHostToDevice));
        }
        CK(cudaMemcpy(clk, &c, sizeof(c), cudaMemcpyHostToDevice));
        return XBG_OK;
    }

    int set_wave_boundary(int slot, const double* St, const double* q, int nrec, const double* times,
                          double t0, double tend, double Trep) override {
        if (slot < 0 || slot > 1 || nrec < 2 || !St || !q) return XBG_ERR_ARG;
        Clock c;
        int rc = read_clock(c);
        if (rc) return rc;
        int phys = slot == 0 ? c.cur_slot : (c.cur_slot ^ 1);
        size_t ns = (size_t)nrec * K.nt * K.ny, nq = (size_t)nrec * 4 * K.ny;
        if (ns > slot_cap) {   // (re)allocate both slots; the step graph is re-captured
            for (int k = 0; k < 2; k++) {
                R* a; R* b;
                if ((rc = alloc(&a, ns)) || (rc = alloc(&b, nq))) return rc;
                if (S.stfile[k]) {
                    CK(cudaMemcpy(a, S.stfile[k], slot_cap * sizeof(R), cudaMemcpyDeviceToDevice));
                    CK(cudaMemcpy(b, S.qfile[k], slot_cap / K.nt * 4 * sizeof(R), cudaMemcpyDeviceToDevice));
                }
                S.stfile[k] = a; S.qfile[k] = b;
            }
            slot_cap = ns;
            drop_graph();
        }
        std::vector<R> hs(ns), hq(nq);
        for (size_t j = 0; j < ns; j++) hs[j] = (R)St[j];
        for (size_t j = 0; j < nq; j++) hq[j] = (R)q[j];
        CK(cudaMemcpy(S.stfile[phys], hs.data(), ns * sizeof(R), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(S.qfile[phys], hq.data(), nq * sizeof(R), cudaMemcpyHostToDevice));
        if (times) {
            if (nrec > XBG_MAX_SERIES) return XBG_ERR_ARG;
            CK(cudaMemcpy(ser->wavet, times, nrec * sizeof(double), cudaMemcpyHostToDevice));
        }
        k_set_slot<R><<<1, 1, 0, st>>>(clk, slot, nrec, t0, tend, Trep);
        launches++;
        CK(cudaGetLastError());
        CK(cudaStreamSynchronize(st));
        return XBG_OK;
    }

    int set_series(int which, const double* t, const double* a, const double* b, int n) override {
        if (n < 2 || n > XBG_MAX_SERIES) return XBG_ERR_ARG;
        Clock c;
        int rc = read_clock(c);
        if (rc) return rc;
        if (which == 0) {
            CK(cudaMemcpy(ser->slt, t, n * sizeof(double), cudaMemcpyHostToDevice));
            CK(cudaMemcpy(ser->sla, a, n * sizeof(double), cudaMemcpyHostToDevice));
            CK(cudaMemcpy(ser->slb, b, n * sizeof(double), cudaMemcpyHostToDevice));
            c.nsl = n; c.SLstep = 1;
        } else {
            CK(cudaMemcpy(ser->wt, t, n * sizeof(double), cudaMemcpyHostToDevice));
            CK(cudaMemcpy(ser->wa, a, n * sizeof(double), cudaMemcpyHostToDevice));
            CK(cudaMemcpy(ser->wb, b, n * sizeof(double), cudaMemcpyHostToDevice));
            c.nwnd = n; c.WNDstep = 1;
        }
        CK(cudaMemcpy(clk, &c, sizeof(c), cudaMemcpyHostToDevice));
        return XBG_OK;
    }

    void drop_graph() {
        if (gexec) { cudaGraphExecDestroy(gexec); gexec = nullptr; }
        if (graph) { cudaGraphDestroy(graph); graph = nullptr; }
        if (seg_exec) { cudaGraphExecDestroy(seg_exec); seg_exec = nullptr; }
        if (seg_graph) { cudaGraphDestroy(seg_graph); seg_graph = nullptr; }
        seg_key[12] = nullptr;
    }

    // one coupled step: the body of mainloopGPU (Wave_gpu.cu:620-757).  In
    // the step graph the boundary kernels (St in time, ubnd1D) form a branch
    // beside the dispersion kernel, which reads neither's outputs; the rows
    // pass joins it.  A profiled step runs every kernel in order.
    int enqueue_step(Prof* pf = nullptr) {
        int n = 0;
        n += launch_step_begin(S, K, ser, nwave, st, pf);
        if (K.swave == 1 && !pf) {
            cudaEventRecord(ev_fork, st);
            cudaStreamWaitEvent(side, ev_fork, 0);
            n += launch_wavebnd(S, K, ser, side, nullptr, 0);
            if (K.flow == 1) n += launch_ubnd(S, K, ser, side, nullptr);
            cudaEventRecord(ev_join, side);
            n += launch_wave(S, K, st, nullptr, ev_join, wave_maps(), wave_cpt(), wide());
        } else {
            if (K.swave == 1) n += launch_wavebnd(S, K, ser, st, pf, 0);
            if (K.flow == 1) n += launch_ubnd(S, K, ser, st, pf);
            if (K.swave == 1) n += launch_wave(S, K, st, pf, nullptr, wave_maps(), wave_cpt(), wide());
        }
        if (K.flow == 1) n += launch_flow(S, K, st, pf, flow_variant == 1, wide(), vec());
        if (P.sedtrans == 1) n += launch_sed(S, K, st, pf, wide(), vec());
        if (K.means) n += launch_means(S, K, st, pf);
        return n;
    }

    int profile_step(float* ms, const char** names, int* n) {
        Prof pf;
        pf.st = st;
        for (int k = 0; k < 65; k++) CK(cudaEventCreate(&pf.ev[k]));
        CK(cudaEventRecord(pf.ev[0], st));
        int nl = enqueue_step(&pf);
        launches += nl;
        CK(cudaGetLastError());
        CK(cudaStreamSynchronize(st));
        int m = std::min(*n, pf.n);
        for (int k = 0; k < m; k++) {
            CK(cudaEventElapsedTime(&ms[k], pf.ev[k], pf.ev[k + 1]));
            if (names) names[k] = pf.name[k];
        }
        *n = m;
        for (int k = 0; k < 65; k++) cudaEventDestroy(pf.ev[k]);
        return XBG_OK;
    }

    int put_records(int slot, int first, int n, const void* St, const void* q) {
        if (slot < 0 || slot > 1 || first < 0 || n < 1 || !St || !q) return XBG_ERR_ARG;
        size_t nyt = (size_t)K.ny * K.nt;
        if ((size_t)(first + n) * nyt > slot_cap) return XBG_ERR_ARG;
        // slot 0 is the chunk in use as of the last call that read the clock
        int phys = slot == 0 ? host_cur_slot : (host_cur_slot ^ 1);
        CK(cudaMemcpyAsync(S.stfile[phys] + (size_t)first * nyt, St, (size_t)n * nyt * sizeof(R),
                           cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(S.qfile[phys] + (size_t)first * 4 * K.ny, q, (size_t)n * 4 * K.ny * sizeof(R),
                           cudaMemcpyHostToDevice, st));
        return XBG_OK;
    }

    int piece(int which) override {
        if (which == 0) clock_stale = true;
        int n = 0;
        switch (which) {
            case 0: n = launch_step_begin(S, K, ser, nwave, st, nullptr); break;
            case 1: if (K.swave == 1) n = launch_wavebnd(S, K, ser, st, nullptr, 1); break;
            case 2: if (K.flow == 1) n = launch_ubnd(S, K, ser, st, nullptr); break;
            case 3:
                if (K.swave == 1) n = launch_wave(S, K, st, nullptr, nullptr, wave_maps(), wave_cpt(), wide());
                break;
            case 4: if (K.flow == 1) n = launch_flow(S, K, st, nullptr, flow_variant == 1, wide(), vec()); break;
            case 5: if (P.sedtrans == 1) n = launch_sed(S, K, st, nullptr, wide(), vec()); break;
            case 6: n = launch_means(S, K, st, nullptr); break;
            default: return XBG_ERR_ARG;
        }
        launches += n;
        CK(cudaGetLastError());
        return XBG_OK;
    }

    int step(int nsteps) override {
        clock_stale = true;
        if (!gexec) {
            CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
            per_step_launches = enqueue_step();
            cudaError_t e = cudaStreamEndCapture(st, &graph);
            if (e != cudaSuccess) { last_err = e; return XBG_ERR_CUDA; }
            CK(cudaGraphInstantiate(&gexec, graph, 0));
        }
        for (int k = 0; k < nsteps; k++) CK(cudaGraphLaunch(gexec, st));
        launches += (int64_t)per_step_launches * nsteps;
        return XBG_OK;
    }

    int get_time(double* t, double* dt, int64_t* n, int* flags) override {
        Clock c;
        int rc = read_clock(c);
        if (rc) return rc;
        if (t) *t = c.totaltime;
        if (dt) *dt = c.dt;
        if (n) *n = c.nstep_total;
        if (flags) *flags = c.flags;
        return c.status;
    }
    // ---- checkpoint / resume: every buffer that carries state from one step
    // to the next, in one host buffer behind a header that names the grid
    struct StateHeader {
        uint64_t magic, version;
        int32_t precision, nx, ny, nt;
        uint64_t slot_cap, nwave, nflow, total;
    };
    static constexpr uint64_t STATE_MAGIC = 0x5854535447425858ull;   // "XXBGTSTX"
    template <class F> void state_regions(F&& f) {
        const size_t C = (size_t)S.C, nt = (size_t)K.nt, ny = (size_t)K.ny;
        for (int k = 0; k < NF2D; k++) f((void*)S.f[k], C * sizeof(R));
        f((void*)S.wetu, C * sizeof(int));
        f((void*)S.wetv, C * sizeof(int));
        f((void*)S.umeanbnd, ny * sizeof(R));
        for (int k = 0; k < 2; k++) {
            f((void*)ee_buf[k], C * nt * sizeof(R));
            f((void*)rr_buf[k], C * nt * sizeof(R));
            f((void*)zsold_buf[k], C * sizeof(R));
        }
        f((void*)S.St, ny * nt * sizeof(R));
        f((void*)S.part_wave, (size_t)nwave * sizeof(R));
        f((void*)S.part_flow, (size_t)2 * step_begin_blocks(K) * sizeof(R));
        f((void*)clk, sizeof(Clock));
        f((void*)ser, sizeof(Series));
        for (int k = 0; k < 2; k++) {
            f((void*)S.stfile[k], slot_cap * sizeof(R));
            f((void*)S.qfile[k], slot_cap / nt * 4 * sizeof(R));
        }
    }
    int state_bytes(size_t* n) override {
        if (!n) return XBG_ERR_ARG;
        size_t t = sizeof(StateHeader);
        state_regions([&](void*, size_t b) { t += b; });
        *n = t;
        return XBG_OK;
    }
    int save_state(void* dst, size_t n) override {
        size_t need = 0;
        state_bytes(&need);
        if (!dst || n < need) return XBG_ERR_ARG;
        if (ext) CK(cudaStreamSynchronize(ext));
        CK(cudaStreamSynchronize(st));
        StateHeader h{STATE_MAGIC, 1, precision, K.nx, K.ny, K.nt, slot_cap, (uint64_t)nwave,
                      (uint64_t)step_begin_blocks(K), need};
        std::memcpy(dst, &h, sizeof(h));
        unsigned char* p = (unsigned char*)dst + sizeof(h);
        int rc = XBG_OK;
        state_regions([&](void* d, size_t b) {
            if (b && !rc && cudaMemcpy(p, d, b, cudaMemcpyDeviceToHost) != cudaSuccess) rc = XBG_ERR_CUDA;
            p += b;
        });
        return rc;
    }
    int load_state(const void* src, size_t n) override {
        if (!src || n < sizeof(StateHeader)) return XBG_ERR_ARG;
        StateHeader h;
        std::memcpy(&h, src, sizeof(h));
        if (h.magic != STATE_MAGIC || h.version != 1 || h.precision != precision || h.nx != K.nx ||
            h.ny != K.ny || h.nt != K.nt || h.nwave != (uint64_t)nwave ||
            h.nflow != (uint64_t)step_begin_blocks(K) || h.total != n)
            return XBG_ERR_ARG;
        if (ext) CK(cudaStreamSynchronize(ext));
        CK(cudaStreamSynchronize(st));
        // a batch's tables hold this handle's slot pointers: a batch scenario
        // takes only snapshots whose boundary slots fit its own
        if (ext && h.slot_cap != slot_cap) return XBG_ERR_STATE;
        if (h.slot_cap != slot_cap) {   // the boundary slots of the saved run
            for (int k = 0; k < 2; k++) {
                if (S.stfile[k]) { release(S.stfile[k]); S.stfile[k] = nullptr; }
                if (S.qfile[k]) { release(S.qfile[k]); S.qfile[k] = nullptr; }
                if (h.slot_cap) {
                    int rc;
                    if ((rc = alloc(&S.stfile[k], h.slot_cap)) || (rc = alloc(&S.qfile[k], h.slot_cap / K.nt * 4)))
                        return rc;
                }
            }
            slot_cap = h.slot_cap;
        }
        drop_graph();   // re-captured with the buffers as they are now
        const unsigned char* p = (const unsigned char*)src + sizeof(h);
        int rc = XBG_OK;
        state_regions([&](void* d, size_t b) {
            if (b && !rc && cudaMemcpy(d, p, b, cudaMemcpyHostToDevice) != cudaSuccess) rc = XBG_ERR_CUDA;
            p += b;
        });
        clock_stale = true;
        if (!rc) {
            Clock c;
            rc = read_clock(c);
        }
        return rc;
    }

    // the clock copied to host memory in stream order, without waiting
    int get_time_async(void* dst) override {
        if (!dst) return XBG_ERR_ARG;
        CK(cudaMemcpyAsync(dst, clk, sizeof(Clock), cudaMemcpyDeviceToHost, st));
        return XBG_OK;
    }
    int clock_decode(const void* src, double* t, double* dt, int64_t* n, int* flags) override {
        if (!src) return XBG_ERR_ARG;
        Clock c;
        std::memcpy(&c, src, sizeof(c));
        host_cur_slot = c.cur_slot;   // as a synchronous read would
        host_par = c.par;
        if (t) *t = c.totaltime;
        if (dt) *dt = c.dt;
        if (n) *n = c.nstep_total;
        if (flags) *flags = c.flags;
        return c.status;
    }
    int set_time(double t, double dt, double wdt) override {
        Clock c;
        int rc = read_clock(c);
        if (rc) return rc;
        c.totaltime = t; c.dt = dt; c.wdt = (float)wdt;
        c.halt = 0;
        c.do_sed = (P.sedtrans == 1 && t >= P.sedstart) ? 1 : 0;
        CK(cudaMemcpy(clk, &c, sizeof(c), cudaMemcpyHostToDevice));
        return XBG_OK;
    }
    int output_done() override { launch_output_done(S, K, st); launches += 2; CK(cudaGetLastError()); return XBG_OK; }
    int reset_means() override { launch_reset_means(S, st); launches += 2; CK(cudaGetLastError()); return XBG_OK; }
    int mass(double* w, double* s, double* b) override {
        CK(cudaMemsetAsync(mass_buf, 0, 3 * sizeof(double), st));
        launch_mass(S, P.dx * P.dx, mass_buf, st);
        launches++;
        double h[3];
        CK(cudaMemcpyAsync(h, mass_buf, sizeof(h), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        *w = h[0]; *s = h[1]; *b = h[2];
        return XBG_OK;
    }
    int sync() override { CK(cudaStreamSynchronize(st)); return XBG_OK; }
    void* stream() override { return (void*)st; }
    int profile(float* ms, const char** names, int* n) override { return profile_step(ms, names, n); }
    int set_forcing(const void* const* f0, const void* const* f1, double w, int rescale) override {
        Forcing6<R> a, b;
        for (int c = 0; c < 6; c++) {
            if (!f0[c] || !f1[c]) return XBG_ERR_ARG;
            a.p[c] = (const R*)f0[c];
            b.p[c] = (const R*)f1[c];
        }
        k_set_forcing<R><<<(S.C + 255) / 256, 256, 0, st>>>(S, ee_buf[0], ee_buf[1], rr_buf[0], rr_buf[1], a, b, (R)w,
                                                            rescale);
        launches++;
        CK(cudaGetLastError());
        return XBG_OK;
    }
    int set_variant(int phase, int variant) override {
        int* slot = nullptr;
        if (phase == XBG_PHASE_WAVE) {
            if (variant < 0 || variant > 2 || (variant >= 1 && !maps_ok)) return XBG_ERR_ARG;
            slot = &wave_variant;
        } else if (phase == XBG_PHASE_FLOW) {
            if (variant < 0 || variant > 1) return XBG_ERR_ARG;
            slot = &flow_variant;
        } else if (phase == XBG_PHASE_TILE) {
            const int vw = sizeof(R) == 4 ? 4 : 2;   // cells per 16-byte segment
            if (variant < 0 || variant > 2 || (variant == 2 && K.nx % vw != 0)) return XBG_ERR_ARG;
            slot = &tile_variant;
        } else {
            return XBG_ERR_ARG;
        }
        if (variant != *slot) {
            CK(cudaStreamSynchronize(st));
            *slot = variant;
            drop_graph();
        }
        return XBG_OK;
    }
    int get_variant(int phase, int* variant) override {
        if (!variant) return XBG_ERR_ARG;
        if (phase == XBG_PHASE_WAVE) *variant = wave_maps() ? wave_variant : 0;
        else if (phase == XBG_PHASE_FLOW) *variant = flow_variant;
        else if (phase == XBG_PHASE_TILE) *variant = tile_variant;
        else return XBG_ERR_ARG;
        return XBG_OK;
    }
    int put_wave_records(int slot, int first, int n, const void* St, const void* q) override {
        return put_records(slot, first, n, St, q);
    }
    // k coupled steps whose wave sub-step is the forcing f0 + (j/k)(f1 - f0)
    // (the rescale at j = k): per step the dt/clock pass, ubnd1D, the forcing,
    // flow, sediment and means -- the sequence a caller gets from
    // xbg_compute_dt, xbg_flow_boundary, xbg_set_wave_forcing, xbg_flow_step,
    // xbg_sediment_step, xbg_accumulate_means, captured once per (f0, f1, k)
    // as one graph and replayed.
    int forcing_steps(const void* const* f0, const void* const* f1, int k) override {
        Forcing6<R> a, b;
        for (int c = 0; c < 6; c++) {
            if (!f0[c] || !f1[c]) return XBG_ERR_ARG;
            a.p[c] = (const R*)f0[c];
            b.p[c] = (const R*)f1[c];
        }
        bool same = seg_exec && seg_key[12] == (const void*)(intptr_t)k;
        for (int c = 0; c < 6 && same; c++) same = seg_key[c] == f0[c] && seg_key[6 + c] == f1[c];
        if (!same) {
            if (seg_exec) { cudaGraphExecDestroy(seg_exec); seg_exec = nullptr; }
            if (seg_graph) { cudaGraphDestroy(seg_graph); seg_graph = nullptr; }
            CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
            int n = 0;
            for (int j = 1; j <= k; j++) {
                n += launch_step_begin(S, K, ser, nwave, st, nullptr);
                if (K.flow == 1) n += launch_ubnd(S, K, ser, st, nullptr);
                k_set_forcing<R><<<(S.C + 255) / 256, 256, 0, st>>>(S, ee_buf[0], ee_buf[1], rr_buf[0], rr_buf[1],
                                                                    a, b, (R)((double)j / k), j == k ? 1 : 0);
                n++;
                if (K.flow == 1) n += launch_flow(S, K, st, nullptr, flow_variant == 1, wide(), vec());
                if (P.sedtrans == 1) n += launch_sed(S, K, st, nullptr, wide(), vec());
                n += launch_means(S, K, st, nullptr);
            }
            cudaError_t e = cudaStreamEndCapture(st, &seg_graph);
            if (e != cudaSuccess) { last_err = e; return XBG_ERR_CUDA; }
            CK(cudaGraphInstantiate(&seg_exec, seg_graph, 0));
            for (int c = 0; c < 6; c++) { seg_key[c] = f0[c]; seg_key[6 + c] = f1[c]; }
            seg_key[12] = (const void*)(intptr_t)k;
            seg_launches = n;
        }
        clock_stale = true;
        CK(cudaGraphLaunch(seg_exec, st));
        launches += seg_launches;
        return XBG_OK;
    }
};

// A batch of scenarios advanced together: N ordinary handles (their
// buffers, clocks and boundary data), device tables of their Dev/Konst and
// per-scenario extras, one work list per tile shape, and one CUDA graph of
// a whole batched step (one launch per kernel for all scenarios).
template <class R>
struct Batch : public xbg_batch {
    std::vector<Handle<R>*> hs;
    Dev<R>* dS = nullptr;
    Konst<R>* dK = nullptr;
    BatchAux* dA = nullptr;
    Clock* dclk = nullptr;
    int2* ditems[BS_N] = {};
    BatchLaunch L{};
    std::vector<Dev<R>> hS;
    std::vector<cudaEvent_t> evs;
    cudaStream_t st = nullptr;
    cudaStream_t side = nullptr;          // the boundary kernels' branch of the step graph
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    int per_step = 0;
    int64_t nlaunch = 0;
    cudaError_t last_err = cudaSuccess;
    int nt = 0, swave = 0, flow = 0, sedtrans = 0, roller = 0, means = 0, wci = 0;   // wci: any scenario with wave-current interaction
    WaveMaps* dmaps = nullptr;            // the scenarios' tensor maps (TMA rows pass), if every scenario has them
    int wave_variant = XBG_WAVE_VARIANT_DEFAULT;   // 1, 2: TMA rows pass (when dmaps), 0: thread-copied tiles
    const WaveMaps* wave_maps() const { return wave_variant >= 1 ? dmaps : nullptr; }
    int wave_cpt() const { return wave_variant == 2 ? 2 : 1; }
    int tile_variant = 0;   // the pointwise passes over 32 x 8 (0) or 64 x 4 (1) tiles
    bool wide() const { return tile_variant == 1; }
    int flow_variant = XBG_FLOW_VARIANT_DEFAULT;   // 1: momentum steps in one pass, 0: two
    // surrogate-assisted stepping: forcing planes per scenario, graphs of
    // forced segments by length, judge accumulators
    std::vector<ForcingPair<R>> hfp;
    ForcingPair<R>* dfp = nullptr;
    std::vector<ErrPair<R>> hep;
    ErrPair<R>* dep = nullptr;
    double* dacc = nullptr;
    std::map<int, cudaGraphExec_t> seg_exec;
    std::map<int, cudaGraph_t> seg_graph;
    std::map<int, int> seg_n;

    ~Batch() override {
        if (gexec) cudaGraphExecDestroy(gexec);
        if (graph) cudaGraphDestroy(graph);
        for (auto e : evs) cudaEventDestroy(e);
        for (auto& kv : seg_exec) cudaGraphExecDestroy(kv.second);
        for (auto& kv : seg_graph) cudaGraphDestroy(kv.second);
        cudaFree(dS); cudaFree(dK); cudaFree(dA); cudaFree(dclk); cudaFree(dmaps);
        cudaFree(dfp); cudaFree(dep); cudaFree(dacc);
        for (int k = 0; k < BS_N; k++) cudaFree(ditems[k]);
        for (auto p : hs) delete p;
        if (ev_fork) cudaEventDestroy(ev_fork);
        if (ev_join) cudaEventDestroy(ev_join);
        if (side) cudaStreamDestroy(side);
        if (st) cudaStreamDestroy(st);
    }

    int setup(const xbg_params* ps, int ns, int prec) {
        n = ns;
        CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        CK(cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking));
        CK(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&ev_join, cudaEventDisableTiming));
        for (int s = 0; s < ns; s++) {
            const xbg_params& p = ps[s];
            if (s == 0) {
                nt = p.ntheta; swave = p.swave; flow = p.flow; sedtrans = p.sedtrans; roller = p.roller; means = p.means;
            } else if (p.ntheta != nt || p.swave != swave || p.flow != flow || p.sedtrans != sedtrans ||
                       p.roller != roller || p.means != means) {
                return XBG_ERR_ARG;   // one kernel sequence for the whole batch
            }
            if (p.wci != 0.0) wci = 1;
            auto* hp = new Handle<R>();
            hs.push_back(hp);
            h.push_back(hp);
            hp->batch_owned = true;
            hp->ext = st;
            int rc = hp->setup(&p, prec);
            if (rc) return rc;
        }
        // tables
        std::vector<Konst<R>> hK(ns);
        std::vector<BatchAux> hA(ns);
        hS.resize(ns);
        std::vector<int2> it[BS_N];
        for (int s = 0; s < ns; s++) {
            Handle<R>& H = *hs[s];
            hS[s] = H.S; hK[s] = H.K;
            const int nx = H.K.nx, ny = H.K.ny, C = nx * ny;
            hA[s].ser = H.ser;
            hA[s].nflow = std::min((C + 255) / 256, 32);   // within the handle's 2 * step_begin_blocks partials
            hA[s].nwave = H.nwave;
            hA[s].ubnd_threads = ubnd_threads(H.K);
            hA[s].scen = s;
            auto add = [&](int sh, int bx, int by) { it[sh].push_back(make_int2(s, bx | (by << 16))); };
            for (int by = 0; by < (ny + 7) / 8; by++)
                for (int bx = 0; bx < (nx + 31) / 32; bx++) add(BS_TILE, bx, by);
            for (int by = 0; by < (ny + 3) / 4; by++)
                for (int bx = 0; bx < (nx + 63) / 64; bx++) add(BS_WIDE, bx, by);
            for (int by = 0; by < (ny - 2 + 7) / 8; by++)
                for (int bx = 0; bx < (nx + 31) / 32; bx++) add(BS_WROWS, bx, by);
            for (int b = 0; b < (C + 255) / 256; b++) add(BS_LIN, b, 0);
            add(BS_ONE, 0, 0);
            for (int b = 0; b < (ny * nt + 255) / 256; b++) add(BS_BND, b, 0);
            for (int b = 0; b < hA[s].nflow; b++) add(BS_DT, b, 0);
        }
        bool all_maps = true;
        for (int s = 0; s < ns; s++) all_maps = all_maps && hs[s]->maps_ok;
        if (all_maps) {
            std::vector<WaveMaps> hm(ns);
            for (int s = 0; s < ns; s++) hm[s] = hs[s]->maps;
            CK(cudaMalloc(&dmaps, ns * sizeof(WaveMaps)));
            CK(cudaMemcpy(dmaps, hm.data(), ns * sizeof(WaveMaps), cudaMemcpyHostToDevice));
        }
        CK(cudaMalloc(&dS, ns * sizeof(Dev<R>)));
        CK(cudaMalloc(&dK, ns * sizeof(Konst<R>)));
        CK(cudaMalloc(&dA, ns * sizeof(BatchAux)));
        CK(cudaMalloc(&dclk, ns * sizeof(Clock)));
        CK(cudaMemcpy(dK, hK.data(), ns * sizeof(Konst<R>), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(dA, hA.data(), ns * sizeof(BatchAux), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(dS, hS.data(), ns * sizeof(Dev<R>), cudaMemcpyHostToDevice));
        int dev = 0, sms = 148;
        CK(cudaGetDevice(&dev));
        CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        const int per_sm[BS_N] = {8, dmaps ? 4 : 3, 8, 2, 8, 8, 8};   // resident-block targets per SM
        for (int k = 0; k < BS_N; k++) {
            CK(cudaMalloc(&ditems[k], std::max<size_t>(1, it[k].size()) * sizeof(int2)));
            CK(cudaMemcpy(ditems[k], it[k].data(), it[k].size() * sizeof(int2), cudaMemcpyHostToDevice));
            L.items[k] = ditems[k];
            L.n[k] = (int)it[k].size();
            L.grid[k] = std::max(1, std::min(L.n[k], sms * per_sm[k]));
        }
        evs.resize(ns);
        for (int s = 0; s < ns; s++) CK(cudaEventCreateWithFlags(&evs[s], cudaEventDisableTiming));
        hfp.assign(ns, ForcingPair<R>{});
        hep.assign(ns, ErrPair<R>{});
        CK(cudaMalloc(&dfp, ns * sizeof(ForcingPair<R>)));
        CK(cudaMemset(dfp, 0, ns * sizeof(ForcingPair<R>)));
        CK(cudaMalloc(&dep, ns * sizeof(ErrPair<R>)));
        CK(cudaMalloc(&dacc, 2 * ns * sizeof(double)));
        for (auto* hp : hs) CK(cudaStreamSynchronize(hp->st));
        return XBG_OK;
    }

    BatchTab<R> tab() const { return BatchTab<R>{dS, dK, dA}; }

    // dt/clock pass, boundaries and the wave solver of one batched step
    int enqueue_waves(const BatchTab<R>& T, Prof* pf) {
        int k = 0;
        k += launch_step_begin_batch(T, L, st, pf);
        if (swave == 1 && !pf) {   // the boundary kernels beside the dispersion kernel, as for one handle
            cudaEventRecord(ev_fork, st);
            cudaStreamWaitEvent(side, ev_fork, 0);
            k += launch_wavebnd_batch(T, L, side, nullptr);
            if (flow == 1) k += launch_ubnd_batch(T, L, side, nullptr);
            cudaEventRecord(ev_join, side);
            k += launch_wave_batch(T, L, nt, roller, wci, st, nullptr, ev_join, wave_maps(), wave_cpt(), wide());
        } else {
            if (swave == 1) k += launch_wavebnd_batch(T, L, st, pf);
            if (flow == 1) k += launch_ubnd_batch(T, L, st, pf);
            if (swave == 1)
                k += launch_wave_batch(T, L, nt, roller, wci, st, pf, nullptr, wave_maps(), wave_cpt(), wide());
        }
        return k;
    }
    // flow, sediment and means of one batched step
    int enqueue_rest(const BatchTab<R>& T, Prof* pf) {
        int k = 0;
        if (flow == 1) k += launch_flow_batch(T, L, st, pf, flow_variant == 1, wide());
        if (sedtrans == 1) k += launch_sed_batch(T, L, st, pf, wide());
        if (means) k += launch_means_batch(T, L, st, pf);
        return k;
    }
    int enqueue(Prof* pf) {
        BatchTab<R> T = tab();
        int k = enqueue_waves(T, pf);
        return k + enqueue_rest(T, pf);
    }

    // order the batch after the scenarios' own streams and refresh the
    // scenario table (a boundary upload may have moved a scenario's slots)
    int prepare() {
        for (int s = 0; s < n; s++) {
            CK(cudaEventRecord(evs[s], hs[s]->st));
            CK(cudaStreamWaitEvent(st, evs[s], 0));
            hS[s] = hs[s]->S;
        }
        CK(cudaMemcpyAsync(dS, hS.data(), n * sizeof(Dev<R>), cudaMemcpyHostToDevice, st));
        return XBG_OK;
    }

    int advance(int nsteps) override {
        int rc = prepare();
        if (rc) return rc;
        if (!gexec) {
            CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
            per_step = enqueue(nullptr);
            cudaError_t e = cudaStreamEndCapture(st, &graph);
            if (e != cudaSuccess) { last_err = e; return XBG_ERR_CUDA; }
            CK(cudaGraphInstantiate(&gexec, graph, 0));
        }
        for (int k = 0; k < nsteps; k++) CK(cudaGraphLaunch(gexec, st));
        nlaunch += (int64_t)per_step * nsteps;
        return XBG_OK;
    }

    int status(double* t, double* dt, int64_t* nstep, int* flags, int* stt) override {
        k_gather_clocks<R><<<n, 64, 0, st>>>(dS, n, dclk);
        CK(cudaGetLastError());
        std::vector<Clock> c(n);
        CK(cudaMemcpyAsync(c.data(), dclk, n * sizeof(Clock), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        for (int s = 0; s < n; s++) {
            if (t) t[s] = c[s].totaltime;
            if (dt) dt[s] = c[s].dt;
            if (nstep) nstep[s] = c[s].nstep_total;
            if (flags) flags[s] = c[s].flags;
            if (stt) stt[s] = c[s].status;
        }
        return XBG_OK;
    }

    int sync() override { CK(cudaStreamSynchronize(st)); return XBG_OK; }
    void* stream() override { return (void*)st; }
    int64_t launches() override { return nlaunch; }

    void drop_segments() {
        for (auto& kv : seg_exec) cudaGraphExecDestroy(kv.second);
        for (auto& kv : seg_graph) cudaGraphDestroy(kv.second);
        seg_exec.clear(); seg_graph.clear(); seg_n.clear();
    }
    int set_grid(int shape, int blocks) override {
        if (shape < 0 || shape >= BS_N || blocks < 1) return XBG_ERR_ARG;
        L.grid[shape] = std::min(blocks, std::max(1, L.n[shape]));
        if (gexec) { cudaGraphExecDestroy(gexec); gexec = nullptr; }
        if (graph) { cudaGraphDestroy(graph); graph = nullptr; }
        drop_segments();
        return XBG_OK;
    }

    int set_variant(int phase, int variant) override {
        int* slot = nullptr;
        if (phase == XBG_PHASE_WAVE) {
            if (variant < 0 || variant > 2 || (variant >= 1 && !dmaps)) return XBG_ERR_ARG;
            slot = &wave_variant;
        } else if (phase == XBG_PHASE_FLOW) {
            if (variant < 0 || variant > 1) return XBG_ERR_ARG;
            slot = &flow_variant;
        } else if (phase == XBG_PHASE_TILE) {
            if (variant < 0 || variant > 1) return XBG_ERR_ARG;
            slot = &tile_variant;
        } else {
            return XBG_ERR_ARG;
        }
        if (variant != *slot) {
            CK(cudaStreamSynchronize(st));
            *slot = variant;
            if (gexec) { cudaGraphExecDestroy(gexec); gexec = nullptr; }
            if (graph) { cudaGraphDestroy(graph); graph = nullptr; }
            drop_segments();
        }
        return XBG_OK;
    }
    int get_variant(int phase, int* variant) override {
        if (!variant) return XBG_ERR_ARG;
        if (phase == XBG_PHASE_WAVE) *variant = wave_maps() ? wave_variant : 0;
        else if (phase == XBG_PHASE_FLOW) *variant = flow_variant;
        else if (phase == XBG_PHASE_TILE) *variant = tile_variant;
        else return XBG_ERR_ARG;
        return XBG_OK;
    }
    int set_wave_mode(int s, int mode) override {
        if (s < 0 || s >= n || mode < XBG_WAVE_PLAIN || mode > XBG_WAVE_FALLBACK) return XBG_ERR_ARG;
        if (mode == XBG_WAVE_FORCED && !hfp[s].f0[0]) return XBG_ERR_STATE;   // no forcing planes yet
        k_set_wave_mode<<<1, 1, 0, st>>>(hs[s]->clk, mode == XBG_WAVE_FORCED ? 1 : 0, mode == XBG_WAVE_FALLBACK);
        nlaunch++;
        CK(cudaGetLastError());
        return XBG_OK;
    }
    int set_forcing(int s, const void* const* f0, const void* const* f1) override {
        if (s < 0 || s >= n || !f0 || !f1) return XBG_ERR_ARG;
        ForcingPair<R> fp;
        for (int c = 0; c < 6; c++) {
            if (!f0[c] || !f1[c]) return XBG_ERR_ARG;
            fp.f0[c] = (const R*)f0[c];
            fp.f1[c] = (const R*)f1[c];
        }
        hfp[s] = fp;
        CK(cudaMemcpyAsync(dfp + s, &hfp[s], sizeof(fp), cudaMemcpyHostToDevice, st));
        return XBG_OK;
    }
    // k coupled steps of every scenario: scenarios in forced mode take the
    // wave sub-step of step j from f0 + (j/k)(f1 - f0) (rescaled at j = k),
    // the others run the wave solver; one CUDA graph per k, replayed
    int forced_segment(int k) override {
        if (k < 1 || k > 100000) return XBG_ERR_ARG;
        int rc = prepare();
        if (rc) return rc;
        if (!seg_exec.count(k)) {
            BatchTab<R> T = tab();
            CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
            int cnt = 0;
            for (int j = 1; j <= k; j++) {
                cnt += enqueue_waves(T, nullptr);
                kb_set_forcing<R><<<L.grid[BS_LIN], 256, 0, st>>>(T, dfp, (R)((double)j / k), j == k ? 1 : 0,
                                                                   L.items[BS_LIN], L.n[BS_LIN]);
                cnt++;
                cnt += enqueue_rest(T, nullptr);
            }
            cudaGraph_t g = nullptr;
            cudaError_t e = cudaStreamEndCapture(st, &g);
            if (e != cudaSuccess) { last_err = e; return XBG_ERR_CUDA; }
            cudaGraphExec_t x = nullptr;
            CK(cudaGraphInstantiate(&x, g, 0));
            seg_graph[k] = g; seg_exec[k] = x; seg_n[k] = cnt;
        }
        CK(cudaGraphLaunch(seg_exec[k], st));
        nlaunch += seg_n[k];
        return XBG_OK;
    }
    int rel_err(int field, const void* const* pred, double* err) override {
        if (!pred || !err) return XBG_ERR_ARG;
        int rc = prepare();
        if (rc) return rc;
        for (int s = 0; s < n; s++) {
            size_t m = 0;
            const R* f = hs[s]->field_ptr(field, &m, 0);
            if (!f || m != (size_t)hs[s]->S.C || field == XBG_F_EE || field == XBG_F_RR || field == XBG_F_ZSOLD)
                return XBG_ERR_ARG;
            hep[s] = ErrPair<R>{f, (const R*)pred[s]};
        }
        CK(cudaMemcpyAsync(dep, hep.data(), n * sizeof(ErrPair<R>), cudaMemcpyHostToDevice, st));
        CK(cudaMemsetAsync(dacc, 0, 2 * n * sizeof(double), st));
        kb_rel_err<R><<<L.grid[BS_LIN], 256, 0, st>>>(tab(), dep, dacc, L.items[BS_LIN], L.n[BS_LIN]);
        nlaunch++;
        CK(cudaGetLastError());
        std::vector<double> h(2 * n);
        CK(cudaMemcpyAsync(h.data(), dacc, 2 * n * sizeof(double), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        for (int s = 0; s < n; s++)
            err[s] = pred[s] ? std::sqrt(h[2 * s]) / std::max(std::sqrt(h[2 * s + 1]), 1e-30) : -1.0;
        return XBG_OK;
    }

    int profile(float* ms, const char** names, int* nk) override {
        int rc = prepare();
        if (rc) return rc;
        Prof pf;
        pf.st = st;
        for (int k = 0; k < 65; k++) CK(cudaEventCreate(&pf.ev[k]));
        CK(cudaEventRecord(pf.ev[0], st));
        nlaunch += enqueue(&pf);
        CK(cudaGetLastError());
        CK(cudaStreamSynchronize(st));
        int m = std::min(*nk, pf.n);
        for (int k = 0; k < m; k++) {
            CK(cudaEventElapsedTime(&ms[k], pf.ev[k], pf.ev[k + 1]));
            if (names) names[k] = pf.name[k];
        }
        *nk = m;
        for (int k = 0; k < 65; k++) cudaEventDestroy(pf.ev[k]);
        return XBG_OK;
    }
};

}  // namespace

// ------------------------------------------------------------------ C ABI
extern "C" {

int xbg_create(const xbg_params* p, int precision, xbg_handle** out) {
    if (!p || !out) return XBG_ERR_ARG;
    *out = nullptr;
    xbg_handle* h = nullptr;
    int rc;
    if (precision == XBG_FP32) { auto* q = new Handle<float>(); rc = q->setup(p, precision); h = q; }
    else if (precision == XBG_FP64) { auto* q = new Handle<double>(); rc = q->setup(p, precision); h = q; }
    else return XBG_ERR_ARG;
    if (rc) { delete h; return rc; }
    *out = h;
    return XBG_OK;
}
int xbg_destroy(xbg_handle* h) {
    if (h && h->batch_owned) return XBG_ERR_STATE;   // freed with its batch
    delete h;
    return XBG_OK;
}
int xbg_init_state(xbg_handle* h, const void* zb, double zs0, double zs1) { return h ? h->init_state(zb, zs0, zs1) : XBG_ERR_ARG; }
int xbg_field_count(const xbg_handle* h, int f, size_t* n) { return h ? const_cast<xbg_handle*>(h)->field_count(f, n) : XBG_ERR_ARG; }
int xbg_set_field(xbg_handle* h, int f, const void* p, size_t n) { return h ? h->set_field(f, p, n) : XBG_ERR_ARG; }
int xbg_get_field(xbg_handle* h, int f, void* p, size_t n) { return h ? h->get_field(f, p, n) : XBG_ERR_ARG; }
int xbg_field_device_ptr(xbg_handle* h, int f, void** p, size_t* n) { return h ? h->device_ptr(f, p, n) : XBG_ERR_ARG; }
int xbg_set_wave_boundary(xbg_handle* h, int slot, const double* St, const double* q, int nrec,
                          const double* times, double t0, double tend, double Trep) {
    return h ? h->set_wave_boundary(slot, St, q, nrec, times, t0, tend, Trep) : XBG_ERR_ARG;
}
int xbg_set_sealevel(xbg_handle* h, const double* t, const double* a, const double* b, int n) { return h ? h->set_series(0, t, a, b, n) : XBG_ERR_ARG; }
int xbg_set_wind(xbg_handle* h, const double* t, const double* a, const double* b, int n) { return h ? h->set_series(1, t, a, b, n) : XBG_ERR_ARG; }
int xbg_compute_dt(xbg_handle* h) { return h ? h->piece(0) : XBG_ERR_ARG; }
int xbg_wave_boundary(xbg_handle* h) { return h ? h->piece(1) : XBG_ERR_ARG; }
int xbg_flow_boundary(xbg_handle* h) { return h ? h->piece(2) : XBG_ERR_ARG; }
int xbg_wave_step(xbg_handle* h) { return h ? h->piece(3) : XBG_ERR_ARG; }
int xbg_flow_step(xbg_handle* h) { return h ? h->piece(4) : XBG_ERR_ARG; }
int xbg_sediment_step(xbg_handle* h) { return h ? h->piece(5) : XBG_ERR_ARG; }
int xbg_accumulate_means(xbg_handle* h) { return h ? h->piece(6) : XBG_ERR_ARG; }
int xbg_step(xbg_handle* h) { return h ? h->step(1) : XBG_ERR_ARG; }
int xbg_advance(xbg_handle* h, int n) { return h ? h->step(n) : XBG_ERR_ARG; }
int xbg_get_time(xbg_handle* h, double* t, double* dt, int64_t* n, int* flags) { return h ? h->get_time(t, dt, n, flags) : XBG_ERR_ARG; }
int xbg_get_time_async(xbg_handle* h, void* dst) { return h ? h->get_time_async(dst) : XBG_ERR_ARG; }
int xbg_state_bytes(xbg_handle* h, size_t* bytes) { return h ? h->state_bytes(bytes) : XBG_ERR_ARG; }
int xbg_save_state(xbg_handle* h, void* dst, size_t bytes) { return h ? h->save_state(dst, bytes) : XBG_ERR_ARG; }
int xbg_load_state(xbg_handle* h, const void* src, size_t bytes) {
    return h ? h->load_state(src, bytes) : XBG_ERR_ARG;
}
int xbg_clock_decode(xbg_handle* h, const void* src, double* t, double* dt, int64_t* n, int* flags) {
    return h ? h->clock_decode(src, t, dt, n, flags) : XBG_ERR_ARG;
}
int xbg_output_done(xbg_handle* h) { return h ? h->output_done() : XBG_ERR_ARG; }
int xbg_reset_means(xbg_handle* h) { return h ? h->reset_means() : XBG_ERR_ARG; }
int xbg_set_time(xbg_handle* h, double t, double dt, double wdt) { return h ? h->set_time(t, dt, wdt) : XBG_ERR_ARG; }
int xbg_sync(xbg_handle* h) { return h ? h->sync() : XBG_ERR_ARG; }
int xbg_fetch_fields(xbg_handle* h, const int* fields, int n, void* const* host) {
    return h ? h->fetch(fields, n, host) : XBG_ERR_ARG;
}
int xbg_launch_count(const xbg_handle* h, int64_t* n) { if (!h || !n) return XBG_ERR_ARG; *n = h->launches; return XBG_OK; }
int xbg_get_stream(xbg_handle* h, void** s) { if (!h || !s) return XBG_ERR_ARG; *s = h->stream(); return XBG_OK; }
int xbg_set_kernel_variant(xbg_handle* h, int phase, int variant) {
    return h ? h->set_variant(phase, variant) : XBG_ERR_ARG;
}
int xbg_get_kernel_variant(xbg_handle* h, int phase, int* variant) {
    return h ? h->get_variant(phase, variant) : XBG_ERR_ARG;
}
int xbg_profile_step(xbg_handle* h, float* ms, const char** names, int* n) {
    if (!h || !ms || !n) return XBG_ERR_ARG;
    return h->profile(ms, names, n);
}
int xbg_put_wave_records(xbg_handle* h, int slot, int first, int n, const void* St, const void* q) {
    return h ? h->put_wave_records(slot, first, n, St, q) : XBG_ERR_ARG;
}
int xbg_mass(xbg_handle* h, double* w, double* s, double* b) { return h ? h->mass(w, s, b) : XBG_ERR_ARG; }
int xbg_set_wave_forcing(xbg_handle* h, const void* const* f0, const void* const* f1, double w, int rescale) {
    return (h && f0 && f1) ? h->set_forcing(f0, f1, w, rescale) : XBG_ERR_ARG;
}
int xbg_forcing_steps(xbg_handle* h, const void* const* f0, const void* const* f1, int k) {
    return (h && f0 && f1 && k >= 1 && k <= 100000) ? h->forcing_steps(f0, f1, k) : XBG_ERR_ARG;
}

int xbg_batch_create(const xbg_params* p, int n, int precision, xbg_batch** out) {
    if (!p || !out || n < 1 || n > XBG_MAX_BATCH || (precision != XBG_FP32 && precision != XBG_FP64))
        return XBG_ERR_ARG;
    *out = nullptr;
    xbg_batch* b = nullptr;
    int rc;
    if (precision == XBG_FP32) { auto* q = new Batch<float>(); b = q; rc = q->setup(p, n, precision); }
    else { auto* q = new Batch<double>(); b = q; rc = q->setup(p, n, precision); }
    if (rc) { delete b; return rc; }
    *out = b;
    return XBG_OK;
}
int xbg_batch_destroy(xbg_batch* b) { delete b; return XBG_OK; }
int xbg_batch_scenario(xbg_batch* b, int s, xbg_handle** h) {
    if (!b || !h || s < 0 || s >= b->n) return XBG_ERR_ARG;
    *h = b->h[s];
    return XBG_OK;
}
int xbg_batch_advance(xbg_batch* b, int nsteps) { return (b && nsteps >= 0) ? b->advance(nsteps) : XBG_ERR_ARG; }
int xbg_batch_status(xbg_batch* b, double* t, double* dt, int64_t* nstep, int* flags, int* status) {
    return b ? b->status(t, dt, nstep, flags, status) : XBG_ERR_ARG;
}
int xbg_batch_sync(xbg_batch* b) { return b ? b->sync() : XBG_ERR_ARG; }
int xbg_batch_get_stream(xbg_batch* b, void** s) { if (!b || !s) return XBG_ERR_ARG; *s = b->stream(); return XBG_OK; }
int xbg_batch_profile_step(xbg_batch* b, float* ms, const char** names, int* n) {
    if (!b || !ms || !n) return XBG_ERR_ARG;
    return b->profile(ms, names, n);
}
int xbg_batch_set_kernel_variant(xbg_batch* b, int phase, int variant) {
    return b ? b->set_variant(phase, variant) : XBG_ERR_ARG;
}
int xbg_batch_get_kernel_variant(xbg_batch* b, int phase, int* variant) {
    return b ? b->get_variant(phase, variant) : XBG_ERR_ARG;
}
int xbg_batch_set_wave_mode(xbg_batch* b, int s, int mode) { return b ? b->set_wave_mode(s, mode) : XBG_ERR_ARG; }
int xbg_batch_set_forcing(xbg_batch* b, int s, const void* const* f0, const void* const* f1) {
    return b ? b->set_forcing(s, f0, f1) : XBG_ERR_ARG;
}
int xbg_batch_forced_segment(xbg_batch* b, int k) { return b ? b->forced_segment(k) : XBG_ERR_ARG; }
int xbg_batch_rel_err(xbg_batch* b, int field, const void* const* pred, double* err) {
    return b ? b->rel_err(field, pred, err) : XBG_ERR_ARG;
}
int xbg_batch_set_grid(xbg_batch* b, int shape, int blocks) { return b ? b->set_grid(shape, blocks) : XBG_ERR_ARG; }
int xbg_batch_launch_count(xbg_batch* b, int64_t* n) { if (!b || !n) return XBG_ERR_ARG; *n = b->launches(); return XBG_OK; }

}  // extern "C"
