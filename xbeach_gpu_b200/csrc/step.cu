// step.cu -- the per-step control that the reference runs on the host
// (mainloopGPU dt logic Wave_gpu.cu:620-698, wavebnd Wavestep.cu:512-753,
// flowbnd Wave_gpu.cu:1020-1103) moved onto the device, plus ubnd1D and the
// running means.
//
//   k_step_begin  FLOWDT per block (Wave_kernel.cu:161) over hh; the last block
//                 to finish reduces all block minima (true global minimum,
//                 not the first 32 block minima of finalminmaxKernel), applies
//                 the dt limiter and output-time snapping, advances the clock,
//                 the wave-boundary record cursor and chunk slots, and the
//                 sea-level / wind cursors, and interpolates St in time.
//                 No block waits on another: the last block is found with an
//                 atomic counter.  A halted step (end time, pending output,
//                 error) sets clk->halt and every later kernel of the step
//                 returns at once.  The same pass checks that hh and zs
//                 are finite everywhere; a NaN or inf sets XBG_ERR_NAN,
//                 which halts this and every later step of the handle
//                 (the reference exits on a NaN dt, Wave_gpu.cu:642-647).
//   k_ubnd       ubnd1D / ubnd1Dnowaves (Flow_kernel.cu:167-242, 332-408) in
//                 one block: the column mean of the pre-kernel uu, then the
//                 ix = 0 column.
//   k_means       addavg_var x6 + max_var (Wave_gpu.cu:731-757).
#include "xbg_common.cuh"
#include "../../include/xbg.h"

namespace xbg {

__device__ __forceinline__ double interptime(double next, double prev, double timenext, double time) {
    return prev + (time) / (timenext) * (next - prev);   // tools.cpp:22-25
}

__device__ __forceinline__ void advance_cursor(const double* t, int n, int& cur, double now) {
    if (cur < n && t[cur] - now < 0.0) cur++;
    if (cur >= n) cur = n - 1;
}

template <class R>
__device__ void wavebnd_cursor(Clock& c, const Konst<R>& K, const Series* ser);

template <class R>
__device__ void finalize_scalar(const Dev<R>& S, const Konst<R>& K, const Series* ser, R mflow, R mwave) {
    Clock& c = *S.clk;
    c.halt = 1;
    if (c.status != XBG_OK) return;
    if (c.flags & (XBG_FLAG_OUTPUT_DUE | XBG_FLAG_ENDED)) return;
    if (!(c.totaltime < K.endtime)) { c.flags |= XBG_FLAG_ENDED; return; }
    c.nstep++;
    c.nstep_total++;
    R wd = (R)c.dt;                                  // wdt = dt, Wave_gpu.cu:622
    double ndt = (double)mflow * 0.5;
    // 0, inf or NaN (the reference's "Model crashed!", Wave_gpu.cu:642-647),
    // or negative: a block of the dt pass saw a non-finite hh or zs
    if (!(ndt > 0.0) || isinf(ndt)) { c.status = XBG_ERR_NAN; return; }
    if (K.swave == 1 && c.totaltime > 0.0) {
        double dtwave = (double)mwave * 0.5;
        ndt = cmin(ndt, dtwave);
    }
    R diffdt = (R)(ndt - (double)wd);
    if (DM<R>::fabs(diffdt) / wd > 0.1) ndt = (double)wd * (1 + (double)(diffdt / DM<R>::fabs(diffdt)) * 0.1);
    double nextstop = cmin(c.nextoutputtime, K.endtime);
    if (ceil((nextstop - c.totaltime) / ndt) > 0.0) ndt = (nextstop - c.totaltime) / ceil((nextstop - c.totaltime) / ndt);
    c.wdt = (float)wd;
    c.dt = ndt;
    c.totaltime = c.totaltime + ndt;
    double t = c.totaltime;
    c.par ^= 1;
    c.do_sed = (K.sedtrans == 1 && t >= K.sedstart) ? 1 : 0;
    if (c.nextoutputtime - t <= ndt * 0.001 && K.outputtimestep > 0) c.flags |= XBG_FLAG_OUTPUT_DUE;
    if (t >= K.endtime) c.flags |= XBG_FLAG_ENDED;
    c.halt = 0;
    if (K.swave == 1) wavebnd_cursor(c, K, ser);   // wavebnd follows the clock
}

// 16-byte vectors of the state's fields (their bases are 16-byte aligned)
template <class R> struct Vec16;
template <> struct Vec16<float> { using T = float4; static constexpr int N = 4; };
template <> struct Vec16<double> { using T = double2; static constexpr int N = 2; };

template <class R>
__device__ __forceinline__ void b_step_begin(const Dev<R>& S, const Konst<R>& K, const Series* ser, int nflow,
                                             int nwave, const int bi, const int nb) {
    __shared__ R red[8], rw[8];
    __shared__ int last;
    int tid = threadIdx.x;
    R m = (R)3.0e38f;
    {   // FLOWDT: max of hh first (16-byte loads, two of each field in flight
        // per thread), one sqrt per thread
        using VT = typename Vec16<R>::T;
        constexpr int N = Vec16<R>::N;
        union U { VT v; R a[N]; };
        const R* hh = S.f[HH];
        const R* zs = S.f[ZS];
        const VT* hv = reinterpret_cast<const VT*>(hh);
        const VT* zv = reinterpret_cast<const VT*>(zs);
        const int nv = S.C / N;
        const int stride = nb * blockDim.x;
        R hmax = (R)0;
        // health check of the state: a NaN or infinite depth or water level
        // anywhere (the sum of every value read times 0 is 0 only if each is finite)
        R probe = (R)0;
        auto take = [&](const U& h, const U& z) {
#pragma unroll
            for (int k = 0; k < N; k++) {
                hmax = DM<R>::fmax(hmax, h.a[k]);
                probe = probe + (h.a[k] * (R)0 + z.a[k] * (R)0);
            }
        };
        int j = bi * blockDim.x + tid;
        for (; j + stride < nv; j += 2 * stride) {
            U h0, h1, z0, z1;
            h0.v = __ldg(hv + j); h1.v = __ldg(hv + j + stride);
            z0.v = __ldg(zv + j); z1.v = __ldg(zv + j + stride);
            take(h0, z0);
            take(h1, z1);
        }
        if (j < nv) {
            U h0, z0;
            h0.v = __ldg(hv + j); z0.v = __ldg(zv + j);
            take(h0, z0);
        }
        // the cells past the last whole vector
        if (bi == 0 && tid < S.C - nv * N) {
            const int i = nv * N + tid;
            hmax = DM<R>::fmax(hmax, ld(hh + i));
            probe = probe + (ld(hh + i) * (R)0 + ld(zs + i) * (R)0);
        }
        // cfl*dx/sqrt(g*hh) decreases with hh, so its minimum is at the deepest cell
        if (hmax > (R)0) m = K.cfl * K.dx / (DM<R>::sqrt((R)9.81f * hmax));
        // a non-finite value makes this block's minimum negative, which the
        // min reductions carry to the clock pass (no valid limit is negative)
        if (!(probe == (R)0)) m = (R)-1;
    }
    // this block's share of the wave kernel's per-block WAVEDT minima
    R mwv = (R)3.0e38f;
    for (int j = bi * blockDim.x + tid; j < nwave; j += nb * blockDim.x)
        mwv = DM<R>::fmin(mwv, ld(S.part_wave + j));
    for (int o = 16; o > 0; o >>= 1) {
        m = DM<R>::fmin(m, __shfl_xor_sync(0xffffffffu, m, o));
        mwv = DM<R>::fmin(mwv, __shfl_xor_sync(0xffffffffu, mwv, o));
    }
    if ((tid & 31) == 0) { red[tid >> 5] = m; rw[tid >> 5] = mwv; }
    __syncthreads();
    if (tid == 0) {
        R b = red[0], bw = rw[0];
        for (int w = 1; w < (int)(blockDim.x >> 5); w++) { b = DM<R>::fmin(b, red[w]); bw = DM<R>::fmin(bw, rw[w]); }
        S.part_flow[bi] = b;
        S.part_flow[nb + bi] = bw;
        __threadfence();
        unsigned prev = atomicAdd(S.counter, 1u);
        last = (prev == nb - 1);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    // ---- last block: global minima, clock, boundaries
    R mf = (R)3.0e38f, mw = (R)3.0e38f;
    for (int j = tid; j < nflow; j += blockDim.x) {
        mf = DM<R>::fmin(mf, ((volatile R*)S.part_flow)[j]);
        mw = DM<R>::fmin(mw, ((volatile R*)S.part_flow)[nflow + j]);
    }
    for (int o = 16; o > 0; o >>= 1) {
        mf = DM<R>::fmin(mf, __shfl_xor_sync(0xffffffffu, mf, o));
        mw = DM<R>::fmin(mw, __shfl_xor_sync(0xffffffffu, mw, o));
    }
    __syncthreads();
    if ((tid & 31) == 0) { red[tid >> 5] = mf; rw[tid >> 5] = mw; }
    __syncthreads();
    if (tid == 0) {
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) { mf = DM<R>::fmin(mf, red[w]); mw = DM<R>::fmin(mw, rw[w]); }
        *S.counter = 0;
        finalize_scalar(S, K, ser, mf, mw);
    }
}
template <class R>
__global__ void __launch_bounds__(256) k_step_begin(Dev<R> S, Konst<R> K, const Series* ser, int nflow, int nwave) {
    b_step_begin<R>(S, K, ser, nflow, nwave, blockIdx.x, gridDim.x);
}
template <class R>
__global__ void __launch_bounds__(256) kb_step_begin(BatchTab<R> T, const int2* items, int n) {
    batch_items<R>(T, items, n, [&](const Dev<R>& S, const Konst<R>& K, const BatchAux& A, int bx, int) {
        b_step_begin<R>(S, K, A.ser, A.nflow, A.nwave, bx, A.nflow);
    });
}

// wavebnd's record cursor and chunk slot (Wavestep.cu:512-700, 684-695),
// Trep and sigm of the record in use.  Sets halt on an error.
template <class R>
__device__ void wavebnd_cursor(Clock& c, const Konst<R>& K, const Series* ser) {
    double t = c.totaltime;
    int cs = c.cur_slot;
    if (!c.slot_valid[cs]) { c.status = XBG_ERR_STATE; c.halt = 1; return; }
    if (K.wavebndtype == 1) {
        int n = c.slot_nrec[cs];
        if (c.WAVstep < n && ser->wavet[c.WAVstep] - t < 0.0) c.WAVstep++;
        if (c.WAVstep >= n) { c.status = XBG_ERR_BOUNDARY; c.halt = 1; return; }
        c.nwbndstep = c.WAVstep - 1;
        c.timenext_w = ser->wavet[c.WAVstep] - ser->wavet[c.WAVstep - 1];
        c.timesincelast_w = t - ser->wavet[c.WAVstep - 1];
    } else {
        if (c.slot_tend[cs] - t < 0.0) {
            if (!c.slot_valid[cs ^ 1]) { c.status = XBG_ERR_BOUNDARY; c.halt = 1; return; }
            c.slot_valid[cs] = 0;
            cs ^= 1;
            c.cur_slot = cs;
            c.flags |= XBG_FLAG_NEED_BOUNDARY;
        }
        double cap = (double)(c.slot_nrec[cs] - 2);
        c.nwbndstep = (int)cmin(floor((t - c.slot_t0[cs]) / K.dtbc), cap);
        c.timenext_w = K.dtbc;
        c.timesincelast_w = t - (c.nwbndstep * K.dtbc + c.slot_t0[cs]);
    }
    R Trep = (R)c.slot_Trep[cs];
    c.Trep = (double)Trep;
    c.sigm = (double)(R)(2 * XBG_PI / (double)Trep);
}

template <class R>
__global__ void k_wavebnd_cursor(Dev<R> S, Konst<R> K, const Series* ser) {
    if (!S.clk->halt) wavebnd_cursor(*S.clk, K, ser);
}

// St interpolation in time (Wavestep.cu:703-741), one thread per (iy, bin).
template <class R>
__device__ __forceinline__ void b_wavebnd_interp(const Dev<R>& S, const Konst<R>& K, const int bix, const int biy) {
    const Clock& c = *S.clk;
    if (halted(&c)) return;
    int j = bix * blockDim.x + threadIdx.x;
    int nyt = K.ny * K.nt;
    if (j >= nyt) return;
    int cs = c.cur_slot, nb = c.nwbndstep;
    const R* sf = S.stfile[cs];
    R so = sf[j + (size_t)nb * nyt];
    R sn = sf[j + (size_t)(nb + 1) * nyt];
    S.St[j] = (R)interptime((double)sn, (double)so, c.timenext_w, c.timesincelast_w);
}
XBG_KERNELS(wavebnd_interp)

template <class R>
__device__ __forceinline__ void b_ubnd(const Dev<R>& S, const Konst<R>& K, const Series* ser, const int nthr) {
    Clock* clk = S.clk;
    if (halted(clk)) return;
    const int nx = K.nx, ny = K.ny;
    if (threadIdx.x == 0) {   // flowbnd sea level and wind (Wave_gpu.cu:1020-1103)
        Clock& c = *clk;
        double t = c.totaltime;
        advance_cursor(ser->slt, c.nsl, c.SLstep, t);
        int s = c.SLstep;
        c.zsbndi = interptime(ser->sla[s], ser->sla[s - 1], ser->slt[s] - ser->slt[s - 1], t - ser->slt[s - 1]);
        c.zsbndn = interptime(ser->slb[s], ser->slb[s - 1], ser->slt[s] - ser->slt[s - 1], t - ser->slt[s - 1]);
        advance_cursor(ser->wt, c.nwnd, c.WNDstep, t);
        s = c.WNDstep;
        c.windu = (double)(R)interptime(ser->wa[s], ser->wa[s - 1], ser->wt[s] - ser->wt[s - 1], t - ser->wt[s - 1]);
        c.windv = (double)(R)interptime(ser->wb[s], ser->wb[s - 1], ser->wt[s] - ser->wt[s - 1], t - ser->wt[s - 1]);
    }
    __shared__ R wsum[32];
    __shared__ R uuavg_s;
    int tid = threadIdx.x;
    R* uu = S.f[UU]; R* zs = S.f[ZS]; R* vv = S.f[VV];
    // column mean of the pre-kernel uu (sequential float sum in the reference;
    // here a tree sum)
    R s = (R)0;
    for (int n = tid; n < ny; n += nthr) s += uu[n * nx];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((tid & 31) == 0) wsum[tid >> 5] = s;
    __syncthreads();
    if (tid == 0) {
        R a = (R)0;
        for (int w = 0; w < (int)(nthr >> 5); w++) a += wsum[w];
        uuavg_s = a / (R)ny;
    }
    __syncthreads();
    R uuavg = uuavg_s;
    R g = K.g, dtf = (R)clk->dt, Trep = (R)clk->Trep;
    R ttime = (R)clk->totaltime, time = (R)clk->timesincelast_w, timenext = (R)clk->timenext_w;
    R zsi = (R)clk->zsbndi, zsn = (R)clk->zsbndn;
    int cs = clk->cur_slot, nb = clk->nwbndstep;
    const R* q = S.qfile[cs];
    for (int iy = tid; iy < ny; iy += nthr) {
        int i = iy * nx, xplus = pp(0, nx);
        R zsbnd = zsi + (zsn - zsi) * (((R)iy) / ((R)ny));
        R zsplus = zs[xplus + iy * nx];
        R hh = ld(S.f[HH] + i);
        R ui, factime;
        if (K.swave == 1) {
            R cats = (R)4.0f;
            factime = (R)1.0f / cats / Trep * dtf;
            R taper = DM<R>::fmin(ttime / (R)100.0f, (R)1.0f);
            R qo = q[iy + (size_t)nb * 4 * ny], qn = q[iy + (size_t)(nb + 1) * 4 * ny];
            R qx = (qo + time / timenext * (qn - qo)) * taper;
            R ht = zsbnd + ld(S.f[ZB] + i);
            ui = qx / ht;
        } else {
            factime = (R)(1.0f / 60.0f) * dtf;   // the literal quotient is a float
            ui = (R)0.0f;
        }
        R ur = (R)-1.0f * DM<R>::sqrt(g / hh) * (zsplus - zsbnd);
        R uumean = factime * uuavg + S.umeanbnd[iy] * ((R)1 - factime);
        S.umeanbnd[iy] = uumean;
        R nu = ((R)2.0f) * ui + ur + uumean;
        R nv = vv[xplus + iy * nx];
        uu[i] = nu;
        zs[i] = zsplus;
        vv[i] = nv;
    }
}
template <class R>
__global__ void __launch_bounds__(1024) k_ubnd(Dev<R> S, Konst<R> K, const Series* ser) {
    b_ubnd<R>(S, K, ser, blockDim.x);
}
// one 1024-thread block per scenario; the column sum runs over the scenario's
// own logical thread count, so it adds in the single-domain kernel's order
template <class R>
__global__ void __launch_bounds__(1024) kb_ubnd(BatchTab<R> T, const int2* items, int n) {
    batch_items<R>(T, items, n, [&](const Dev<R>& S, const Konst<R>& K, const BatchAux& A, int, int) {
        b_ubnd<R>(S, K, A.ser, A.ubnd_threads);
    });
}

template <class R>
__device__ __forceinline__ void b_means(const Dev<R>& S, const Konst<R>& K, const int bix, const int biy) {
    if (halted(S.clk)) return;
    int i = bix * blockDim.x + threadIdx.x;
    if (i >= S.C) return;
    // every load before the first store: the field pointers may alias as far
    // as the compiler knows, so interleaved stores would serialise the loads
    R zs = ld(S.f[ZS] + i), hr = ld(S.f[H] + i), u = ld(S.f[UU] + i), v = ld(S.f[VV] + i);
    R h = ld(S.f[HH] + i), c = ld(S.f[CSED] + i);
    R mH = S.f[HMEAN][i], mu = S.f[UUMEAN][i], mv = S.f[VVMEAN][i], mh = S.f[HHMEAN][i];
    R mz = S.f[ZSMEAN][i], xz = S.f[ZSMAX][i], mc = S.f[CMEAN][i];
    S.f[HMEAN][i] = mH + hr;
    S.f[UUMEAN][i] = mu + u;
    S.f[VVMEAN][i] = mv + v;
    S.f[HHMEAN][i] = mh + h;
    S.f[ZSMEAN][i] = mz + zs;
    S.f[ZSMAX][i] = DM<R>::fmax(xz, zs);
    S.f[CMEAN][i] = mc + c;
}
XBG_KERNELS(means)

// The single-domain running means with 16-byte loads and stores: four float
// (two double) cells per thread, the clock's halt flag read with the loads
// and tested before the stores; the last C mod 4 (2) cells by one more
// thread.  Each field is its own allocation, so every vector is aligned.

template <class R>
__global__ void __launch_bounds__(256) k_means_v(Dev<R> S, Konst<R> K) {
    using VT = typename Vec16<R>::T;
    constexpr int N = Vec16<R>::N;
    union U { VT v; R a[N]; };
    const bool off = halted(S.clk);
    const int nv = S.C / N;
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j < nv) {
        auto L = [&](int f) { U u; u.v = __ldg(reinterpret_cast<const VT*>(S.f[f]) + j); return u; };
        auto M = [&](int f) { U u; u.v = reinterpret_cast<const VT*>(S.f[f])[j]; return u; };
        const U zs = L(ZS), hr = L(H), u = L(UU), v = L(VV), h = L(HH), c = L(CSED);
        U mH = M(HMEAN), mu = M(UUMEAN), mv = M(VVMEAN), mh = M(HHMEAN), mz = M(ZSMEAN), xz = M(ZSMAX),
          mc = M(CMEAN);
        loads_before_here();
        if (off) return;
#pragma unroll
        for (int k = 0; k < N; k++) {
            mH.a[k] = mH.a[k] + hr.a[k];
            mu.a[k] = mu.a[k] + u.a[k];
            mv.a[k] = mv.a[k] + v.a[k];
            mh.a[k] = mh.a[k] + h.a[k];
            mz.a[k] = mz.a[k] + zs.a[k];
            xz.a[k] = DM<R>::fmax(xz.a[k], zs.a[k]);
            mc.a[k] = mc.a[k] + c.a[k];
        }
        auto W = [&](int f, const U& x) { reinterpret_cast<VT*>(S.f[f])[j] = x.v; };
        W(HMEAN, mH); W(UUMEAN, mu); W(VVMEAN, mv); W(HHMEAN, mh); W(ZSMEAN, mz); W(ZSMAX, xz); W(CMEAN, mc);
    } else if (j == nv && !off) {
        for (int i = nv * N; i < S.C; i++) {
            const R zs = S.f[ZS][i];
            S.f[HMEAN][i] += S.f[H][i];
            S.f[UUMEAN][i] += S.f[UU][i];
            S.f[VVMEAN][i] += S.f[VV][i];
            S.f[HHMEAN][i] += S.f[HH][i];
            S.f[ZSMEAN][i] += zs;
            S.f[ZSMAX][i] = DM<R>::fmax(S.f[ZSMAX][i], zs);
            S.f[CMEAN][i] += S.f[CSED][i];
        }
    }
}

template <class R>
__global__ void k_output_done(Dev<R> S, Konst<R> K) {   // Wave_gpu.cu:786-824
    const Clock& c = *S.clk;
    R nd = (R)c.nstep;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < S.C) {
        int ids[6] = {HMEAN, UUMEAN, VVMEAN, HHMEAN, ZSMEAN, CMEAN};
        for (int k = 0; k < 6; k++) S.f[ids[k]][i] = S.f[ids[k]][i] / nd;
    }
}

// nextoutputtime advance after an output (Wave_gpu.cu:789)
template <class R>
__global__ void k_output_clock(Dev<R> S, Konst<R> K) {
    Clock& c = *S.clk;
    c.nextoutputtime = c.nextoutputtime + K.outputtimestep;
    c.flags &= ~XBG_FLAG_OUTPUT_DUE;
}
template <class R>
__global__ void k_reset_clock(Dev<R> S) { S.clk->nstep = 0; }

template <class R>
__global__ void k_reset_means(Dev<R> S) {   // Wave_gpu.cu:894-928
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < S.C) {
        int ids[7] = {HMEAN, UUMEAN, VVMEAN, HHMEAN, ZSMEAN, ZSMAX, CMEAN};
        for (int k = 0; k < 7; k++) S.f[ids[k]][i] = (R)0;
    }
}

template <class R>
__global__ void k_mass(Dev<R> S, double dx2, double* out) {
    __shared__ double r[3][8];
    int tid = threadIdx.x;
    double a = 0, b = 0, c = 0;
    for (int i = blockIdx.x * blockDim.x + tid; i < S.C; i += gridDim.x * blockDim.x) {
        a += (double)S.f[ZS][i];
        b += (double)S.f[CSED][i] * (double)S.f[HH][i];
        c += (double)S.f[ZB][i];
    }
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_xor_sync(0xffffffffu, a, o);
        b += __shfl_xor_sync(0xffffffffu, b, o);
        c += __shfl_xor_sync(0xffffffffu, c, o);
    }
    if ((tid & 31) == 0) { r[0][tid >> 5] = a; r[1][tid >> 5] = b; r[2][tid >> 5] = c; }
    __syncthreads();
    if (tid == 0) {
        a = b = c = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) { a += r[0][w]; b += r[1][w]; c += r[2][w]; }
        atomicAdd(out + 0, a * dx2);
        atomicAdd(out + 1, b * dx2);
        atomicAdd(out + 2, c * dx2);
    }
}

// ---------------------------------------------------------------- launchers
template <class R>
int step_begin_blocks(const Konst<R>& K) {
    int nb = (K.nx * K.ny + 255) / 256;
    // grid-stride, eight blocks (2048 threads) per SM: enough loads in flight
    // to cover the memory latency, and few partials to reduce
    return nb < 8 * 148 ? nb : 8 * 148;
}

template <class R>
int launch_step_begin(const Dev<R>& S, const Konst<R>& K, const Series* ser, int nwave, cudaStream_t st, Prof* pf) {
    int nb = step_begin_blocks(K);
    k_step_begin<R><<<nb, 256, 0, st>>>(S, K, ser, nb, nwave);
    PMARK(pf, "k_step_begin");
    return 1;
}
// logical thread count of the single-domain ubnd launch
template <class R>
int ubnd_threads(const Konst<R>& K) { return K.ny >= 1024 ? 1024 : ((K.ny + 31) / 32) * 32; }

template <class R>
int launch_ubnd(const Dev<R>& S, const Konst<R>& K, const Series* ser, cudaStream_t st, Prof* pf) {
    k_ubnd<R><<<1, ubnd_threads(K), 0, st>>>(S, K, ser);
    PMARK(pf, "k_ubnd");
    return 1;
}
template <class R>
int launch_wavebnd(const Dev<R>& S, const Konst<R>& K, const Series* ser, cudaStream_t st, Prof* pf, int cursor) {
    // in a whole step the dt kernel has already moved the record cursor
    if (cursor) k_wavebnd_cursor<R><<<1, 1, 0, st>>>(S, K, ser);
    int nyt = K.ny * K.nt;
    k_wavebnd_interp<R><<<(nyt + 255) / 256, 256, 0, st>>>(S, K);
    if (cursor) { PMARK(pf, "k_wavebnd"); return 2; }
    PMARK(pf, "k_wavebnd");
    return 1;
}
template <class R>
int launch_means(const Dev<R>& S, const Konst<R>& K, cudaStream_t st, Prof* pf) {
    const int nthr = S.C / Vec16<R>::N + 1;
    k_means_v<R><<<(nthr + 255) / 256, 256, 0, st>>>(S, K);
    PMARK(pf, "k_means");
    return 1;
}
template <class R>
void launch_output_done(const Dev<R>& S, const Konst<R>& K, cudaStream_t st) {
    k_output_done<R><<<(S.C + 255) / 256, 256, 0, st>>>(S, K);
    k_output_clock<R><<<1, 1, 0, st>>>(S, K);
}
template <class R>
void launch_reset_means(const Dev<R>& S, cudaStream_t st) {
    k_reset_means<R><<<(S.C + 255) / 256, 256, 0, st>>>(S);
    k_reset_clock<R><<<1, 1, 0, st>>>(S);
}
template <class R>
void launch_mass(const Dev<R>& S, double dx2, double* out, cudaStream_t st) {
    k_mass<R><<<296, 256, 0, st>>>(S, dx2, out);
}

// the step-control kernels over every scenario of a batch
template <class R>
int launch_step_begin_batch(const BatchTab<R>& T, const BatchLaunch& L, cudaStream_t st, Prof* pf) {
    kb_step_begin<R><<<L.grid[BS_DT], 256, 0, st>>>(T, L.items[BS_DT], L.n[BS_DT]);
    PMARK(pf, "k_step_begin");
    return 1;
}
template <class R>
int launch_wavebnd_batch(const BatchTab<R>& T, const BatchLaunch& L, cudaStream_t st, Prof* pf) {
    kb_wavebnd_interp<R><<<L.grid[BS_BND], 256, 0, st>>>(T, L.items[BS_BND], L.n[BS_BND]);
    PMARK(pf, "k_wavebnd");
    return 1;
}
template <class R>
int launch_ubnd_batch(const BatchTab<R>& T, const BatchLaunch& L, cudaStream_t st, Prof* pf) {
    kb_ubnd<R><<<L.grid[BS_ONE], 1024, 0, st>>>(T, L.items[BS_ONE], L.n[BS_ONE]);
    PMARK(pf, "k_ubnd");
    return 1;
}
template <class R>
int launch_means_batch(const BatchTab<R>& T, const BatchLaunch& L, cudaStream_t st, Prof* pf) {
    kb_means<R><<<L.grid[BS_LIN], 256, 0, st>>>(T, L.items[BS_LIN], L.n[BS_LIN]);
    PMARK(pf, "k_means");
    return 1;
}
#define INST(R)                                                                                   \
    template int step_begin_blocks<R>(const Konst<R>&);                                           \
    template int launch_step_begin<R>(const Dev<R>&, const Konst<R>&, const Series*, int, cudaStream_t, Prof*); \
    template int launch_ubnd<R>(const Dev<R>&, const Konst<R>&, const Series*, cudaStream_t, Prof*);     \
    template int launch_wavebnd<R>(const Dev<R>&, const Konst<R>&, const Series*, cudaStream_t, Prof*, int); \
    template int launch_means<R>(const Dev<R>&, const Konst<R>&, cudaStream_t, Prof*);                   \
    template void launch_output_done<R>(const Dev<R>&, const Konst<R>&, cudaStream_t);            \
    template void launch_reset_means<R>(const Dev<R>&, cudaStream_t);                             \
    template void launch_mass<R>(const Dev<R>&, double, double*, cudaStream_t);                        \
    template int ubnd_threads<R>(const Konst<R>&);                                                \
    template int launch_step_begin_batch<R>(const BatchTab<R>&, const BatchLaunch&, cudaStream_t, Prof*); \
    template int launch_wavebnd_batch<R>(const BatchTab<R>&, const BatchLaunch&, cudaStream_t, Prof*);    \
    template int launch_ubnd_batch<R>(const BatchTab<R>&, const BatchLaunch&, cudaStream_t, Prof*);       \
    template int launch_means_batch<R>(const BatchTab<R>&, const BatchLaunch&, cudaStream_t, Prof*);
INST(float)
INST(double)

}  // namespace xbg
