/*
 * xbg_oracle.cpp -- TEST INFRASTRUCTURE ONLY (see xbg_oracle.h).
 *
 * A plain, loop-by-loop CPU restatement of XBeach_GPU's coupled step, written
 * from the reference sources and instantiated for float (the reference's
 * DECNUM, XBeachGPU.h:37) and for double (the FP64 error oracle).  In the
 * float instantiation every expression keeps the reference's own mix of float
 * and double arithmetic, so the wave functions reproduce wave_CPU.cpp and the
 * flow / sediment functions reproduce the kernels of Flow_kernel.cu and
 * Sediment_kernel.cu as a host compiler evaluates them.
 *
 * Sources followed (reference file:line):
 *   wave step   wave_CPU.cpp (the reference's CPU judge), call order of
 *               wavestepCPU, Wavestep.cu:1169-1302
 *   boundaries  wavebnd Wavestep.cu:512-753, flowbnd Wave_gpu.cu:1020-1103,
 *               ubnd1D Flow_kernel.cu:167-242, ubnd1Dnowaves :332-408
 *   flow step   Flow_kernel.cu kernels in flowstep order, Wave_gpu.cu:1142-1397
 *   sediment    Sediment_kernel.cu kernels in sedimentstep order,
 *               Wave_gpu.cu:1462-1606
 *   time step   Wave_gpu.cu:620-698, FLOWDT/WAVEDT Wave_kernel.cu:161,232
 *   means       Wave_gpu.cu:731-757, Wave_kernel.cu:85-158
 *   init        Wave_gpu.cu:1988-2015, 2519-2551, 2637-2692,
 *               Wavestep.cu:79-86, 355-375
 *
 * Fixed semantics where the reference GPU code races or is undefined (the
 * same choices are made by the CUDA kernels):
 *   1. dt uses the true global minimum (minmaxKernel/finalminmaxKernel reduce
 *      only the first 32 block minima, Wave_gpu.cu:633).
 *   2. vdvdy_fixbnd (Flow_kernel.cu:1076-1100) stores an uninitialised
 *      register into every cell; here vdvdy_adv's values are kept and the
 *      fix is applied only at iy = ny-1 (where eulervstep never writes).
 *   3. ubnd1D averages the pre-kernel uu column (Flow_kernel.cu:207-212).
 *   4. avalanching's neighbour writes (Sediment_kernel.cu:1129-1132) are
 *      gathered per cell in the order a serial launch adds them:
 *      ((-dzby[below] - dzbx[left]) + dzbx) + dzby.
 *   5. In-place boundary-copy kernels read pre-kernel values (corners of
 *      twodimbnd, zblatbnd, CClatbnd).
 *   6. Only threads inside the grid write (ubnd1D and vdvdy_adv lack an iy/ix
 *      bound and write past the arrays when ny or nx is not a multiple of 16).
 * hardlayer and zblatbnd(Sout) (Sediment_kernel.cu:824-879) feed only the
 * bed-load divergence that bedupdate has commented out (:954) and are not
 * evaluated.  longturb's kturb update is `kturb = 0` (:161).
 */
#include "xbg_oracle.h"
#include <cmath>
#include <cstring>
#include <cstdio>
#include <vector>
#include <algorithm>

#define REF_PI 3.14159265   /* the reference's `pi` macro (double literal) */

namespace {

/* ---- math of the element type: float functions for float, double for double */
template <class T> struct M;
template <> struct M<float> {
    static float sqrt(float x) { return sqrtf(x); }
    static float sinh(float x) { return sinhf(x); }
    static float tanh(float x) { return tanhf(x); }
    static float pow(float x, float y) { return powf(x, y); }
    static float exp(float x) { return expf(x); }
    static float log(float x) { return logf(x); }
    static float log10(float x) { return log10f(x); }
    static float cos(float x) { return cosf(x); }
    static float sin(float x) { return sinf(x); }
    static float fabs(float x) { return fabsf(x); }
    static float fmin(float a, float b) { return fminf(a, b); }
    static float fmax(float a, float b) { return fmaxf(a, b); }
    static float atan(float x) { return atanf(x); }
};
template <> struct M<double> {
    static double sqrt(double x) { return ::sqrt(x); }
    static double sinh(double x) { return ::sinh(x); }
    static double tanh(double x) { return ::tanh(x); }
    static double pow(double x, double y) { return ::pow(x, y); }
    static double exp(double x) { return ::exp(x); }
    static double log(double x) { return ::log(x); }
    static double log10(double x) { return ::log10(x); }
    static double cos(double x) { return ::cos(x); }
    static double sin(double x) { return ::sin(x); }
    static double fabs(double x) { return ::fabs(x); }
    static double fmin(double a, double b) { return ::fmin(a, b); }
    static double fmax(double a, double b) { return ::fmax(a, b); }
    static double atan(double x) { return ::atan(x); }
};

/* min/max as wave_CPU.cpp:10-16 defines them (used by the wave functions). */
template <class T> inline T cmax(T a, T b) { return (a < b) ? b : a; }
template <class T> inline T cmin(T a, T b) { return !(b < a) ? a : b; }

/* Clamped neighbour indices, Flow_CPU.cpp:16-70 / Wave_kernel.cu:23-77. */
inline int mm(int i) { return i <= 0 ? 0 : i - 1; }
inline int pp(int i, int n) { return i >= n - 1 ? n - 1 : i + 1; }
inline int mm2(int i) { return i <= 1 ? 0 : i - 2; }
inline int pp2(int i, int n) { return i >= n - 2 ? n - 1 : i + 2; }

/* interptime, tools.cpp:22-25 */
inline double interptime(double next, double prev, double timenext, double time) {
    return prev + (time) / (timenext) * (next - prev);
}

struct Chunk {
    bool valid = false;
    int nrec = 0;
    std::vector<double> times;     /* wavebndtype 1: record times          */
    double t0 = 0, tend = 0, Trep = 0;
    std::vector<double> St, q;     /* [nrec][ntheta][ny], [nrec][4][ny]    */
};

struct Series { std::vector<double> t, a, b; };

}  // namespace

struct xbgo {
    virtual ~xbgo() {}
    virtual int init_state(const void* zb, double zs0, double zs1) = 0;
    virtual int field_count(int f, size_t* n) const = 0;
    virtual int set_field(int f, const void* p, size_t n) = 0;
    virtual int get_field(int f, void* p, size_t n) = 0;
    virtual int compute_dt() = 0;
    virtual int wave_boundary() = 0;
    virtual int flow_boundary() = 0;
    virtual int wave_step() = 0;
    virtual int flow_step() = 0;
    virtual int sediment_step() = 0;
    virtual int means() = 0;
    virtual int output_done() = 0;
    virtual int reset_means() = 0;
    virtual void mass(double* w, double* s, double* b) = 0;

    xbg_params P;
    int precision = XBG_FP32;
    /* host-side time state (mainloopGPU globals) */
    double totaltime = 0, dt = 0, nextoutputtime = 0;
    double wdt = 0;            /* float in the reference (Wave_gpu.cu:78) */
    int64_t nstep = 0;         /* steps since the last output             */
    int64_t nstep_total = 0;
    int flags = 0;
    int status = XBG_OK;
    /* boundary cursors (Wave_gpu.cu:86, 173) */
    int SLstep = 1, WNDstep = 1, WAVstep = 1, nwbndstep = 0;
    double zsbndi = 0, zsbndn = 0, windu = 0, windv = 0;
    double timenext_w = 1, timesincelast_w = 0;   /* ubnd1D interpolation */
    Chunk chunk[2];
    Series sl, wnd;
};

namespace {

template <class T>
struct Oracle : public xbgo {
    int nx, ny, nt, C;
    /* 2-D fields, indexed by xbg_field */
    std::vector<T> F[XBG_F_COUNT];
    std::vector<int> wetu, wetv;
    std::vector<T> theta, cxsth, sxnth;
    std::vector<T> St, qbndold, qbndnew;     /* interpolated boundary rows  */
    T Trep = 0;
    /* per-step temporaries */
    std::vector<T> sigm, kh, sinh2kh, wci, ctheta, xadv, yadv, thadv, Sxx, Sxy,
        Syy, nuhg, viscu, viscv, ududx, vdudy, udvdx, vdvdy, dzsdx, dzsdy, wrk1,
        wrk2, dtflow, ceqbg, Tsg, ua, facero, Sus, Svs, ero, depo, ddzb,
        Eint;
    /* constants of Wave_gpu.cu:93-96 */
    T twopi, aphi, bphi;

    explicit Oracle(const xbg_params* p, int prec) {
        P = *p;
        precision = prec;
        nx = P.nx; ny = P.ny; nt = P.ntheta; C = nx * ny;
        for (int f = 0; f < XBG_F_COUNT; f++) {
            size_t n = (size_t)C;
            if (f == XBG_F_UMEANBND) n = ny;
            if (f == XBG_F_EE || f == XBG_F_RR) n = (size_t)C * nt;
            if (f == XBG_F_WETU || f == XBG_F_WETV) n = 0;
            F[f].assign(n, (T)0);
        }
        wetu.assign(C, 0); wetv.assign(C, 0);
        auto a2 = [&](std::vector<T>& v) { v.assign(C, (T)0); };
        a2(sigm); a2(kh); a2(sinh2kh); a2(wci); a2(Sxx); a2(Sxy); a2(Syy);
        a2(nuhg); a2(viscu); a2(viscv); a2(ududx); a2(vdudy); a2(udvdx);
        a2(vdvdy); a2(dzsdx); a2(dzsdy); a2(wrk1); a2(wrk2); a2(dtflow);
        a2(ceqbg); a2(Tsg); a2(ua); a2(facero); a2(Sus); a2(Svs); a2(ero);
        a2(depo); a2(ddzb); a2(Eint);
        ctheta.assign((size_t)C * nt, (T)0); xadv = ctheta; yadv = ctheta;
        thadv = ctheta;
        St.assign((size_t)ny * nt, (T)0);
        qbndold.assign((size_t)4 * ny, (T)0); qbndnew = qbndold;
        /* theta bins, Wavestep.cu:79-86 */
        theta.resize(nt); cxsth.resize(nt); sxnth.resize(nt);
        for (int i = 0; i < nt; i++) {
            theta[i] = (T)(i * (P.dtheta) + P.thetamin + 0.5f * P.dtheta);
            cxsth[i] = M<T>::cos(theta[i]);
            sxnth[i] = M<T>::sin(theta[i]);
        }
        /* Wave_gpu.cu:93-96 */
        T phi = (T)((1.0f + M<T>::sqrt((T)5.0f)) / 2);
        aphi = 1 / (phi + 1);
        bphi = phi / (phi + 1);
        twopi = 8 * M<T>::atan((T)1.0f);
        nextoutputtime = P.outputtimestep;
    }

    T* f(int id) { return F[id].data(); }
    size_t fsize(int id) const {
        if (id == XBG_F_WETU || id == XBG_F_WETV) return (size_t)C;
        return F[id].size();
    }

    int field_count(int id, size_t* n) const override {
        if (id < 0 || id >= XBG_F_COUNT) return XBG_ERR_ARG;
        *n = fsize(id);
        return XBG_OK;
    }
    int set_field(int id, const void* p, size_t n) override {
        if (id < 0 || id >= XBG_F_COUNT || n != fsize(id)) return XBG_ERR_ARG;
        if (id == XBG_F_WETU || id == XBG_F_WETV) {
            std::memcpy(id == XBG_F_WETU ? wetu.data() : wetv.data(), p, n * sizeof(int));
        } else {
            std::memcpy(F[id].data(), p, n * sizeof(T));
        }
        return XBG_OK;
    }
    int get_field(int id, void* p, size_t n) override {
        if (id < 0 || id >= XBG_F_COUNT || n != fsize(id)) return XBG_ERR_ARG;
        if (id == XBG_F_WETU || id == XBG_F_WETV) {
            std::memcpy(p, id == XBG_F_WETU ? wetu.data() : wetv.data(), n * sizeof(int));
        } else {
            std::memcpy(p, F[id].data(), n * sizeof(T));
        }
        return XBG_OK;
    }

    /* ================================================================ init */
    int init_state(const void* zbp, double zs0, double zs1) override {
        const T* zbin = (const T*)zbp;
        T* zb = f(XBG_F_ZB); T* zs = f(XBG_F_ZS); T* hh = f(XBG_F_HH);
        for (int iy = 0; iy < ny; iy++) {
            f(XBG_F_UMEANBND)[iy] = 0;
            for (int ix = 0; ix < nx; ix++) {
                int i = ix + iy * nx;
                zb[i] = zbin[i];
                /* Wave_gpu.cu:2000-2010 (fnod-1 = iy) */
                double zsbnd = zs0 + (zs1 - zs0) * (iy) / ny;
                zs[i] = cmax((T)zsbnd, (T)(-1 * zb[i]));
                hh[i] = (T)cmax((double)zb[i] + zsbnd, P.eps);
                f(XBG_F_STDEP)[i] = (T)5.0f;   /* no hard-layer file, :2042-2052 */
            }
        }
        /* Wave_gpu.cu:2457-2510: hu, hv, hum, hvm <- hh; zsold <- zs */
        for (int i = 0; i < C; i++) {
            f(XBG_F_HU)[i] = hh[i]; f(XBG_F_HV)[i] = hh[i];
            f(XBG_F_HUM)[i] = hh[i]; f(XBG_F_HVM)[i] = hh[i];
            f(XBG_F_ZSOLD)[i] = zs[i];
        }
        updatezom();
        /* initial dt, Wave_gpu.cu:2648-2679: FLOWDT with 0.5*CFL */
        T cfl = (T)(0.5f * P.CFL);
        double mn = 1e300;
        for (int i = 0; i < C; i++) {
            T v = cfl * (T)P.dx / (M<T>::sqrt((T)9.81f * hh[i]));
            mn = std::min(mn, (double)v);
        }
        dt = (T)mn * 0.5;
        if (dt < 0.00000001) { status = XBG_ERR_DT; return status; }
        wdt = (T)dt;   /* first mainloop iteration sets wdt = dt */
        /* sigm = 2 pi / Trep (set_bnd); ee column 0 = first record */
        if (P.swave == 1) {
            if (!chunk[0].valid) return XBG_ERR_STATE;
            Trep = (T)chunk[0].Trep;
            for (int i = 0; i < C; i++) sigm[i] = (T)(2.0f * REF_PI / Trep);
            T* ee = f(XBG_F_EE);
            for (int t = 0; t < nt; t++)
                for (int iy = 0; iy < ny; iy++)
                    ee[0 + iy * nx + t * C] = (T)chunk[0].St[iy + t * ny];
            /* dispersion_init: cg */
            for (int i = 0; i < C; i++) {
                T k_, c_, kh_, s_, cg_;
                disp(sigm[i], hh[i], k_, c_, kh_, s_, cg_);
                f(XBG_F_CG)[i] = cg_;
            }
        }
        return XBG_OK;
    }

    /* ============================================================ time step */
    int compute_dt() override {
        if (status != XBG_OK) return status;
        nstep++; nstep_total++;
        wdt = (T)dt;                                   /* Wave_gpu.cu:622 */
        const T* hh = f(XBG_F_HH);
        T cfl = (T)P.CFL, dxf = (T)P.dx;
        double mn = 1e300;
        for (int i = 0; i < C; i++) {                  /* FLOWDT */
            T v = cfl * dxf / (M<T>::sqrt((T)9.81f * hh[i]));
            if ((double)v < mn) mn = v;
        }
        double ndt = (T)mn * 0.5;
        /* the CUDA path's dt pass also checks the state itself: a non-finite
         * hh or zs anywhere is the same "model crashed" status */
        const T* zs = f(XBG_F_ZS);
        for (int i = 0; i < C; i++)
            if (!std::isfinite((double)hh[i]) || !std::isfinite((double)zs[i])) ndt = -1.0;
        if (!(ndt > 0.0) || std::isinf(ndt)) {
            status = XBG_ERR_NAN; return status;       /* :642-647 */
        }
        if (P.swave == 1 && totaltime > 0.0) {         /* WAVEDT :651-672 */
            T dth = (T)P.dtheta;
            double mw = 1e300;
            for (int i = 0; i < C; i++) {
                T mindt = (T)9999999.9f;
                for (int t = 0; t < nt; t++)
                    mindt = M<T>::fmin(cfl * dth / M<T>::fabs(ctheta[i + (size_t)t * C]), mindt);
                if ((double)mindt < mw) mw = mindt;
            }
            double dtwave = (T)mw * 0.5;
            ndt = cmin(ndt, dtwave);
        }
        /* :674-679, diffdt is a float */
        T wd = (T)wdt;
        T diffdt = (T)(ndt - wd);
        if (M<T>::fabs(diffdt) / wd > 0.1) ndt = wd * (1 + (diffdt) / M<T>::fabs(diffdt) * 0.1);
        double nextstop = cmin(nextoutputtime, P.endtime);
        if (std::ceil((nextstop - totaltime) / ndt) > 0.0)
            ndt = (nextstop - totaltime) / std::ceil((nextstop - totaltime) / ndt);
        dt = ndt;
        totaltime = totaltime + dt;
        return XBG_OK;
    }

    /* ===================================================== boundary (host) */
    int wave_boundary() override {   /* wavebnd, Wavestep.cu:512-753 */
        if (status != XBG_OK) return status;
        Chunk& ch = chunk[0];
        if (!ch.valid) { status = XBG_ERR_STATE; return status; }
        if (P.wavebndtype == 1) {
            if (WAVstep >= ch.nrec) { status = XBG_ERR_BOUNDARY; return status; }
            if (ch.times[WAVstep] - totaltime < 0.0) WAVstep++;
            if (WAVstep >= ch.nrec) { status = XBG_ERR_BOUNDARY; return status; }
            nwbndstep = WAVstep - 1;
            timenext_w = ch.times[WAVstep] - ch.times[WAVstep - 1];
            timesincelast_w = totaltime - ch.times[WAVstep - 1];
        } else {
            if (ch.tend - totaltime < 0.0) {
                /* next record: the following chunk becomes current */
                if (!chunk[1].valid) { status = XBG_ERR_BOUNDARY; return status; }
                chunk[0] = chunk[1];
                chunk[1] = Chunk();
                flags |= XBG_FLAG_NEED_BOUNDARY;
            }
            Chunk& c0 = chunk[0];
            double cap = (double)(c0.nrec - 2);
            nwbndstep = (int)cmin(std::floor((totaltime - c0.t0) / P.dtbc), cap);
            timenext_w = P.dtbc;
            timesincelast_w = totaltime - (nwbndstep * P.dtbc + c0.t0);
        }
        Chunk& c0 = chunk[0];
        Trep = (T)c0.Trep;
        for (int ni = 0; ni < ny; ni++) {
            for (int it = 0; it < nt; it++) {
                T so = (T)c0.St[ni + it * ny + (size_t)nwbndstep * ny * nt];
                T sn = (T)c0.St[ni + it * ny + (size_t)(nwbndstep + 1) * ny * nt];
                St[ni + it * ny] = (T)interptime(sn, so, timenext_w, timesincelast_w);
            }
            for (int xi = 0; xi < 4; xi++) {
                qbndold[ni + xi * ny] = (T)c0.q[ni + xi * ny + (size_t)nwbndstep * ny * 4];
                qbndnew[ni + xi * ny] = (T)c0.q[ni + xi * ny + (size_t)(nwbndstep + 1) * ny * 4];
            }
        }
        return XBG_OK;
    }

    static void advance_series(const Series& s, int& cur, double t) {
        if (cur < (int)s.t.size() && s.t[cur] - t < 0.0) cur++;
        if (cur >= (int)s.t.size()) cur = (int)s.t.size() - 1;
    }

    int flow_boundary() override {   /* flowbnd, Wave_gpu.cu:1020-1103 */
        if (status != XBG_OK) return status;
        if (sl.t.size() < 2 || wnd.t.size() < 2) { status = XBG_ERR_STATE; return status; }
        advance_series(sl, SLstep, totaltime);
        zsbndi = interptime(sl.a[SLstep], sl.a[SLstep - 1], sl.t[SLstep] - sl.t[SLstep - 1], totaltime - sl.t[SLstep - 1]);
        zsbndn = interptime(sl.b[SLstep], sl.b[SLstep - 1], sl.t[SLstep] - sl.t[SLstep - 1], totaltime - sl.t[SLstep - 1]);
        double timenext = 1, timesincelast = 0;
        if (P.swave == 1) {
            timenext = timenext_w; timesincelast = timesincelast_w;
            ubnd1D((T)totaltime, (T)timesincelast, (T)timenext, (T)zsbndi, (T)zsbndn);
        } else {
            ubnd1Dnowaves((T)totaltime, (T)zsbndi, (T)zsbndn);
        }
        advance_series(wnd, WNDstep, totaltime);
        windu = interptime(wnd.a[WNDstep], wnd.a[WNDstep - 1], wnd.t[WNDstep] - wnd.t[WNDstep - 1], totaltime - wnd.t[WNDstep - 1]);
        windv = interptime(wnd.b[WNDstep], wnd.b[WNDstep - 1], wnd.t[WNDstep] - wnd.t[WNDstep - 1], totaltime - wnd.t[WNDstep - 1]);
        return XBG_OK;
    }

    /* ubnd1D, Flow_kernel.cu:167-242 (column average of the pre-kernel uu) */
    void ubnd1D(T ttime, T time, T timenext, T zsi, T zsn) {
        T* uu = f(XBG_F_UU); T* vv = f(XBG_F_VV); T* zs = f(XBG_F_ZS);
        const T* zb = f(XBG_F_ZB); const T* hh = f(XBG_F_HH);
        T* umean = f(XBG_F_UMEANBND);
        T g = (T)P.g, dtf = (T)dt;
        T uuavg = 0.0f;
        for (int n = 0; n < ny; n++) uuavg = uuavg + uu[0 + n * nx];
        uuavg = uuavg / ny;
        std::vector<T> nu(ny), nz(ny), nv(ny);
        for (int iy = 0; iy < ny; iy++) {
            int i = iy * nx, xplus = pp(0, nx);
            T zsbnd = zsi + (zsn - zsi) * (((T)iy) / ((T)ny));
            T cats = 4.0f;
            T factime = 1.0f / cats / Trep * dtf;
            T taper = M<T>::fmin(ttime / 100.0f, 1.0f);
            T zsplus = zs[xplus + iy * nx];
            T qx = (qbndold[iy] + time / timenext * (qbndnew[iy] - qbndold[iy])) * taper;
            T ht = zsbnd + zb[i];
            T ui = qx / ht;
            T ur = -1.0f * M<T>::sqrt(g / hh[i]) * (zsplus - zsbnd);
            T uumean = factime * uuavg + umean[iy] * (1 - factime);
            umean[iy] = uumean;
            nu[iy] = (2.0f) * ui + ur + uumean;
            nz[iy] = zsplus;
            nv[iy] = vv[xplus + iy * nx];
        }
        for (int iy = 0; iy < ny; iy++) {
            uu[iy * nx] = nu[iy]; zs[iy * nx] = nz[iy]; vv[iy * nx] = nv[iy];
        }
    }

    /* ubnd1Dnowaves, Flow_kernel.cu:332-408 */
    void ubnd1Dnowaves(T ttime, T zsi, T zsn) {
        (void)ttime;
        T* uu = f(XBG_F_UU); T* vv = f(XBG_F_VV); T* zs = f(XBG_F_ZS);
        const T* hh = f(XBG_F_HH);
        T* umean = f(XBG_F_UMEANBND);
        T g = (T)P.g, dtf = (T)dt;
        T uuavg = 0.0f;
        for (int n = 0; n < ny; n++) uuavg = uuavg + uu[0 + n * nx];
        uuavg = uuavg / ny;
        std::vector<T> nu(ny), nz(ny), nv(ny);
        for (int iy = 0; iy < ny; iy++) {
            int i = iy * nx, xplus = pp(0, nx);
            T zsbnd = zsi + (zsn - zsi) * (((T)iy) / ((T)ny));
            T factime = 1.0f / 60.0f * dtf;
            T zsplus = zs[xplus + iy * nx];
            T ui = 0.0f;
            T ur = -1.0f * M<T>::sqrt(g / hh[i]) * (zsplus - zsbnd);
            T uumean = factime * uuavg + umean[iy] * (1 - factime);
            umean[iy] = uumean;
            nu[iy] = (2.0f) * ui + ur + uumean;
            nz[iy] = zsplus;
            nv[iy] = vv[xplus + iy * nx];
        }
        for (int iy = 0; iy < ny; iy++) {
            uu[iy * nx] = nu[iy]; zs[iy * nx] = nz[iy]; vv[iy * nx] = nv[iy];
        }
    }

    /* ========================================================= wave step */
    /* dispersion, wave_CPU.cpp:154-205 */
    void disp(T sg, T h, T& k_, T& c_, T& kh_, T& s2kh_, T& cg_) {
        T g = (T)P.g;
        T L0 = twopi * g / (sg * sg);
        T L1 = L0, L2, errdisp;
        for (int n = 1; n < 200; n++) {
            L2 = (T)(L0 * ::tanh(2 * REF_PI * h / L1));
            errdisp = M<T>::fabs(L2 - L1);
            L1 = (L1 * aphi + L2 * bphi);
            if (errdisp <= 0.0001f) break;
            if (n == 199) {
                L1 = L0 * M<T>::pow(M<T>::tanh(M<T>::pow(sg * sg * h / g, 3.0f / 4.0f)), 2.0f / 3.0f);
                break;
            }
        }
        T kk = (T)(2 * REF_PI / L1);
        k_ = kk;
        T cc = sg / kk;
        c_ = cc;
        T kkhh = cmin(kk * h, (T)10.0f);
        kh_ = kkhh;
        T s2kh = M<T>::sinh(2.0f * kkhh);
        s2kh_ = s2kh;
        cg_ = cc * (0.5f + kkhh / s2kh);
    }

    /* xadvecupwind2CPU (wave_CPU.cpp:367-464) for field q with speed cg */
    void xadv2(const T* q, const T* cg, T* out) {
        const T* uu = f(XBG_F_UU);
        T dx = (T)P.dx;
        T dxplus_i = 1.0f / dx;
        for (int ix = 0; ix < nx; ix++)
            for (int iy = 0; iy < ny; iy++) {
                int i = ix + iy * nx;
                int xm = mm(ix), xp = pp(ix, nx), xp2 = pp2(ix, nx), xm2 = mm2(ix);
                T ccg = cg[i], ccgxmin = cg[xm + iy * nx], ccgxmax = cg[xp + iy * nx];
                T uui = uu[i] * wci[i];
                T uuixmin = uu[xm + iy * nx] * wci[i];
                T uuixmax = uu[xp + iy * nx] * wci[i];
                for (int t = 0; t < nt; t++) {
                    size_t o = (size_t)t * C;
                    T costhet = cxsth[t];
                    T cgx = 0.5f * (ccg * costhet + uui + ccgxmax * costhet + uuixmax);
                    T cgxmin = 0.5f * (ccg * costhet + uui + ccgxmin * costhet + uuixmin);
                    T arrinx, arrminx;
                    if (cgx > 0.0f) {
                        arrinx = (T)(1.5 * q[i + o] - 0.5 * q[xm + iy * nx + o]);
                        if (arrinx < 0.0f) arrinx = q[i + o];
                        arrinx = arrinx * cgx;
                    } else {
                        arrinx = (T)(1.5 * q[xp + iy * nx + o] - 0.5 * q[xp2 + iy * nx + o]);
                        if (arrinx < 0.0f) arrinx = q[xp + iy * nx + o];
                        arrinx = arrinx * cgx;
                    }
                    if (cgxmin > 0.0f) {
                        arrminx = (T)(1.5 * q[xm + iy * nx + o] - 0.5 * q[xm2 + iy * nx + o]);
                        if (arrminx < 0.0f) arrminx = q[xm + iy * nx + o];
                        arrminx = arrminx * cgxmin;
                    } else {
                        arrminx = (T)(1.5 * q[i + o] - 0.5 * q[xp + iy * nx + o]);
                        if (arrminx < 0.0f) arrminx = q[i + o];
                        arrminx = arrminx * cgxmin;
                    }
                    out[i + o] = (arrinx - arrminx) * dxplus_i;
                }
            }
    }

    /* yadvecupwind2CPU (wave_CPU.cpp:467-560) */
    void yadv2(const T* q, const T* cg, T* out) {
        const T* vv = f(XBG_F_VV);
        T dx = (T)P.dx;
        T dxplus_i = 1.0f / dx;
        for (int ix = 0; ix < nx; ix++)
            for (int iy = 0; iy < ny; iy++) {
                int i = ix + iy * nx;
                int ym = mm(iy), yp = pp(iy, ny), ym2 = mm2(iy), yp2 = pp2(iy, ny);
                T ccg = cg[i], ccgymin = cg[ix + ym * nx], ccgymax = cg[ix + yp * nx];
                T vvi = wci[i] * vv[i];
                T vviymin = wci[i] * vv[ix + ym * nx];
                T vviymax = wci[i] * vv[ix + yp * nx];
                for (int t = 0; t < nt; t++) {
                    size_t o = (size_t)t * C;
                    T sinthet = sxnth[t];
                    T cgy = 0.5f * (ccg * sinthet + vvi + ccgymax * sinthet + vviymax);
                    T cgymin = 0.5f * (ccg * sinthet + vvi + ccgymin * sinthet + vviymin);
                    T arriny, arrminy;
                    if (cgy > 0.0f) {
                        arriny = (T)(1.5 * q[i + o] - 0.5 * q[ix + ym * nx + o]);
                        if (arriny < 0.0f) arriny = q[i + o];
                        arriny = arriny * cgy;
                    } else {
                        arriny = (T)(1.5 * q[ix + yp * nx + o] - 0.5 * q[ix + yp2 * nx + o]);
                        if (arriny < 0.0f) arriny = q[ix + yp * nx + o];
                        arriny = arriny * cgy;
                    }
                    if (cgymin > 0.0f) {
                        arrminy = (T)(1.5 * q[ix + ym * nx + o] - 0.5 * q[ix + ym2 * nx + o]);
                        if (arrminy < 0.0f) arrminy = q[ix + ym * nx + o];
                        arrminy = arrminy * cgymin;
                    } else {
                        arrminy = (T)(1.5 * q[i + o] - 0.5 * q[ix + yp * nx + o]);
                        if (arrminy < 0.0f) arrminy = q[i + o];
                        arrminy = arrminy * cgymin;
                    }
                    out[i + o] = (arriny - arrminy) * dxplus_i;
                }
            }
    }

    /* thetaadvecuw2hoCPU (wave_CPU.cpp:706-806) */
    void thadv2(const T* q, T* out) {
        T dth = (T)P.dtheta;
        for (int i = 0; i < C; i++) {
            if (nt > 1) {
                for (int t = 0; t < nt; t++) {
                    int Tm = mm(t), Tp = pp(t, nt), Tm2 = mm2(t), Tp2 = pp2(t, nt);
                    T cthetab, eupw, arrint, arrmint;
                    cthetab = 0.5f * (ctheta[i + (size_t)t * C] + ctheta[i + (size_t)Tp * C]);
                    if (cthetab > 0.0f) {
                        eupw = 1.5f * q[i + (size_t)t * C] - 0.5f * q[i + (size_t)Tm * C];
                        if (eupw < 0.0f) eupw = q[i + (size_t)t * C];
                    } else {
                        eupw = 1.5f * q[i + (size_t)Tp * C] - 0.5f * q[i + (size_t)Tp2 * C];
                        if (eupw < 0.0f) eupw = q[i + (size_t)Tp * C];
                    }
                    arrint = cthetab * eupw;
                    cthetab = 0.5f * (ctheta[i + (size_t)Tm * C] + ctheta[i + (size_t)t * C]);
                    if (cthetab > 0.0f) {
                        eupw = 1.5f * q[i + (size_t)Tm * C] - 0.5f * q[i + (size_t)Tm2 * C];
                        if (eupw < 0.0f) eupw = q[i + (size_t)Tm * C];
                    } else {
                        eupw = 1.5f * q[i + (size_t)t * C] - 0.5f * q[i + (size_t)Tp * C];
                        if (eupw < 0.0f) eupw = q[i + (size_t)t * C];
                    }
                    arrmint = cthetab * eupw;
                    T tt = (arrint - arrmint) / dth;
                    if (t == nt - 1) tt = (0.0f - arrmint) / dth;
                    if (t == 0) tt = (arrint - 0.0f) / dth;
                    out[i + (size_t)t * C] = tt;
                }
            } else {
                out[i] = 0.0f;
            }
        }
    }

    /* eulerupwindCPU (wave_CPU.cpp:811-828) */
    void euler(T* q) {
        T dtf = (T)dt;
        for (size_t j = 0; j < (size_t)C * nt; j++)
            q[j] = q[j] - dtf * (xadv[j] + yadv[j] + thadv[j]);
    }

    /* rollerlatbndCPU (wave_CPU.cpp:830-870), pre-kernel reads */
    void rollerlatbnd(T* q) {
        const T* hh = f(XBG_F_HH);
        T eps = (T)P.eps;
        for (int ix = 0; ix < nx; ix++) {
            for (int t = 0; t < nt; t++) {
                size_t o = (size_t)t * C;
                int i0 = ix, i1 = ix + (ny - 1) * nx;
                T w0 = hh[i0] > eps ? 1.0f : 0.0f;
                T w1 = hh[i1] > eps ? 1.0f : 0.0f;
                T a = q[ix + pp(0, ny) * nx + o] * w0;
                T b = q[ix + mm(ny - 1) * nx + o] * w1;
                q[i0 + o] = a;
                q[i1 + o] = b;
            }
        }
    }

    /* twodimbndnoixCPU / twodimbndCPU (wave_CPU.cpp:1173-1330) */
    void twodimbnd(T* Fv, bool withix) {
        const T* hh = f(XBG_F_HH);
        T eps = (T)P.eps;
        std::vector<T> o(Fv, Fv + C);
        for (int ix = 0; ix < nx; ix++)
            for (int iy = 0; iy < ny; iy++) {
                int i = ix + iy * nx;
                T wet = hh[i] > eps ? 1.0f : 0.0f;
                if (iy == 0) Fv[i] = o[ix + pp(iy, ny) * nx] * wet;
                if (iy == ny - 1) Fv[i] = o[ix + mm(iy) * nx] * wet;
                if (withix && ix == 0) Fv[i] = o[pp(ix, nx) + iy * nx] * wet;
            }
    }

    int wave_step() override {   /* wavestepCPU, Wavestep.cu:1169-1302 */
        if (status != XBG_OK) return status;
        T* ee = f(XBG_F_EE); T* rr = f(XBG_F_RR);
        T* hh = f(XBG_F_HH); T* uu = f(XBG_F_UU); T* vv = f(XBG_F_VV);
        T* k = f(XBG_F_K); T* c = f(XBG_F_C); T* cg = f(XBG_F_CG);
        T* E = f(XBG_F_E); T* H = f(XBG_F_H); T* D = f(XBG_F_D);
        T* R = f(XBG_F_R); T* DR = f(XBG_F_DR);
        T dxf = (T)P.dx, dtf = (T)dt, rho = (T)P.rho, g = (T)P.g;
        T dth = (T)P.dtheta, eps = (T)P.eps;
        /* offshorebndWavCPU, wave_CPU.cpp:24-40 */
        {
            T tt = (T)totaltime;
            T taper = (T)cmin((double)tt / 100.0, 1.0);
            for (int i = 0; i < C; i++) sigm[i] = (T)(2 * REF_PI / Trep);
            for (int t = 0; t < nt; t++)
                for (int iy = 0; iy < ny; iy++)
                    ee[0 + iy * nx + (size_t)t * C] = St[iy + t * ny] * taper;
        }
        /* sanityCPU */
        for (size_t j = 0; j < (size_t)C * nt; j++) ee[j] = cmax(ee[j], (T)0.000f);
        /* dispersionCPU */
        for (int i = 0; i < C; i++) disp(sigm[i], hh[i], k[i], c[i], kh[i], sinh2kh[i], cg[i]);
        /* calcwciCPU */
        for (int i = 0; i < C; i++) wci[i] = (T)P.wci * cmin(hh[i] / (T)P.hwci, (T)1.0f);
        /* slopesCPU + propagthetaCPU (wave_CPU.cpp:226-306) */
        for (int ix = 0; ix < nx; ix++)
            for (int iy = 0; iy < ny; iy++) {
                int i = ix + iy * nx;
                int xm = mm(ix), xp = pp(ix, nx), ym = mm(iy), yp = pp(iy, ny);
                T dhdx = (hh[xp + iy * nx] - hh[xm + iy * nx]) / ((T)(xp - xm) * dxf);
                T dudx = (uu[xp + iy * nx] - uu[xm + iy * nx]) / ((T)(xp - xm) * dxf);
                T dvdx = (vv[xp + iy * nx] - vv[xm + iy * nx]) / ((T)(xp - xm) * dxf);
                T dhdy = (hh[ix + yp * nx] - hh[ix + ym * nx]) / ((T)(yp - ym) * dxf);
                T dudy = (uu[ix + yp * nx] - uu[ix + ym * nx]) / ((T)(yp - ym) * dxf);
                T dvdy = (vv[ix + yp * nx] - vv[ix + ym * nx]) / ((T)(yp - ym) * dxf);
                T s = sigm[i] / M<T>::sinh(2.0f * kh[i]);
                for (int t = 0; t < nt; t++) {
                    T cx = cxsth[t], sx = sxnth[t];
                    T ctht = (s) * (dhdx * sx - dhdy * cx) +
                             wci[i] * (cx * (sx * dudx - cx * dudy) + sx * (sx * dvdx - cx * dvdy));
                    ctheta[i + (size_t)t * C] = cmin(cmax(ctht, (T)(-0.25f * sigm[i])), (T)(0.25f * sigm[i]));
                }
            }
        /* actionCPU */
        for (int t = 0; t < nt; t++)
            for (int i = 0; i < C; i++) ee[i + (size_t)t * C] = ee[i + (size_t)t * C] / sigm[i];
        xadv2(ee, cg, xadv.data());
        yadv2(ee, cg, yadv.data());
        thadv2(ee, thadv.data());
        euler(ee);
        rollerlatbnd(ee);
        /* energyCPU */
        for (int t = 0; t < nt; t++)
            for (int i = 0; i < C; i++) {
                T e = ee[i + (size_t)t * C] * sigm[i];
                ee[i + (size_t)t * C] = cmax(e, (T)0.0f);
            }
        /* energintCPU (wave_CPU.cpp:891-924) */
        T gammax = (T)P.gammax;
        for (int i = 0; i < C; i++) {
            T Etmp = 0.0f;
            T hht = hh[i];
            for (int t = 0; t < nt; t++) Etmp = Etmp + ee[i + (size_t)t * C];
            Etmp = Etmp * dth;
            T Htmp = M<T>::sqrt(Etmp / (rho * g / 8.0f));
            T idiv = cmax((T)1.0f, M<T>::pow(Htmp / (gammax * hht), 2.0f));
            for (int t = 0; t < nt; t++) ee[i + (size_t)t * C] = ee[i + (size_t)t * C] / idiv;
            Htmp = cmin(Htmp, gammax * hht);
            E[i] = (rho * g * Htmp * Htmp) / 8.0f;
            H[i] = Htmp;
        }
        const T* fwm = f(XBG_F_FWM);
        T gam = (T)P.gammaa, alpha = (T)P.alpha, nn = (T)P.n;
        if (P.breakmodel == 1) {
            /* roelvinkCPU (wave_CPU.cpp:927-985) */
            for (int i = 0; i < C; i++) {
                T fac = (T)(8.0 / rho / g);
                T hr = hh[i];
                T etmp = E[i];
                T Htmp = M<T>::sqrt(etmp * fac);
                T Qb = (T)(1.0 - ::exp(cmax(-1.0 * (double)M<T>::pow((Htmp / gam / hr), nn), -100.0)));
                Qb = cmin(Qb, (T)1.0f);
                D[i] = (T)(Qb * 2.0 * alpha / Trep * etmp * Htmp / hr);
                T uorb = (T)(REF_PI * Htmp / (Trep * M<T>::sinh(cmin(k[i] * hr, (T)10.0f))));
                T fw = fwm[i];
                D[i] = (T)(D[i] + 0.66666666f / REF_PI * rho * fw * uorb * uorb * uorb);
            }
        } else {
            /* baldockCPU (wave_CPU.cpp:987-1028) */
            for (int i = 0; i < C; i++) {
                T hb = hh[i], ki = k[i], Htmp = H[i];
                T khh = ki * hb;
                T Hb = (0.88f / ki) * M<T>::tanh(gam * khh / 0.88f);
                T Rr = Hb / cmax(Htmp, (T)0.00001f);
                T Qb = M<T>::exp(-1.0f * Rr * Rr);
                D[i] = 0.25f * alpha * Qb * rho * (1.0f / Trep) * g * (Hb * Hb + Htmp * Htmp);
                T uorb = (T)(REF_PI * Htmp / (Trep * M<T>::sinh(cmin(k[i] * hb, (T)10.0f))));
                D[i] = (T)(D[i] + 0.66666666f / REF_PI * rho * fwm[i] * uorb * uorb * uorb);
            }
        }
        if (P.roller == 1) {   /* Wavestep.cu:1277-1284 */
            xadv2(rr, c, xadv.data());
            yadv2(rr, c, yadv.data());
            thadv2(rr, thadv.data());
            euler(rr);
            rollerlatbnd(rr);
        }
        /* dissipationCPU (wave_CPU.cpp:1030-1092) */
        T beta = (T)P.beta;
        for (int i = 0; i < C; i++) {
            T RR = 0.0f, drr = 0.0f;
            T cc = c[i];
            T uui = uu[i] * wci[i], vvi = vv[i] * wci[i];
            for (int t = 0; t < nt; t++) {
                size_t j = i + (size_t)t * C;
                T cx = cc * cxsth[t] + uui;
                T cy = cc * sxnth[t] + vvi;
                T eet = ee[j];
                T dd = eet * D[i] / cmax(E[i], (T)0.0000001f);
                T rrt;
                if (hh[i] > eps) {
                    rrt = rr[j];
                    T rrd = 2.0f * g * beta * rrt / M<T>::sqrt(cx * cx + cy * cy);
                    eet = cmax(eet - dtf * dd, (T)0.0f);
                    rrt = cmax(rrt + dtf * (dd - rrd), (T)0.0f);
                    drr = drr + rrd;
                } else {
                    eet = 0.0f; rrt = 0.0f; drr = 0.0f;
                }
                RR = RR + rrt;
                ee[j] = eet;
                rr[j] = rrt;
            }
            R[i] = RR * dth;
            DR[i] = drr * dth;
        }
        rollerlatbnd(ee);
        /* meandirCPU (wave_CPU.cpp:1095-1121) */
        T* thm = f(XBG_F_THETAMEAN);
        for (int i = 0; i < C; i++) {
            T sumethet = 0, sume = 0;
            for (int t = 0; t < nt; t++) {
                sume = sume + ee[i + (size_t)t * C];
                sumethet = sumethet + ee[i + (size_t)t * C] * theta[t];
            }
            sume = cmax(sume, (T)0.00001f);
            thm[i] = (sumethet / nt) / (sume / nt);
            E[i] = sume * dth;
            H[i] = M<T>::sqrt(sume * dth / (rho * g / 8));
        }
        /* radstressCPU (wave_CPU.cpp:1123-1162) */
        for (int i = 0; i < C; i++) {
            T n = cg[i] / c[i];
            T sume = 0, txx = 0, txy = 0, tyy = 0, rxx = 0, rxy = 0, ryy = 0;
            for (int t = 0; t < nt; t++) {
                T e = ee[i + (size_t)t * C], r = rr[i + (size_t)t * C];
                T cx = cxsth[t], sx = sxnth[t];
                sume = sume + e;
                txx = txx + ((1.0f + cx * cx) * e);
                tyy = tyy + ((1.0f + sx * sx) * e);
                txy = txy + (sx * cx * e);
                rxx = rxx + ((cx * cx) * r);
                ryy = ryy + ((sx * sx) * r);
                rxy = rxy + (sx * cx * r);
            }
            Sxx[i] = (n * txx - 0.5f * sume) * dth + rxx * dth;
            Syy[i] = (n * tyy - 0.5f * sume) * dth + ryy * dth;
            Sxy[i] = n * txy * dth + rxy * dth;
        }
        /* wavforceCPU (wave_CPU.cpp:1164-1171 ... 1238) */
        T* Fx = f(XBG_F_FX); T* Fy = f(XBG_F_FY);
        for (int ix = 0; ix < nx; ix++)
            for (int iy = 0; iy < ny; iy++) {
                int i = ix + iy * nx;
                int xm = mm(ix), xp = pp(ix, nx), ym = mm(iy), yp = pp(iy, ny);
                T Sxxi = Sxx[i], Sxxr = Sxx[xp + iy * nx], Sxyt = Sxy[ix + yp * nx];
                T Sxytr = Sxy[xp + yp * nx], Sxyb = Sxy[ix + ym * nx], Sxybr = Sxy[xp + ym * nx];
                T Syyi = Syy[i], Syyt = Syy[ix + yp * nx], Sxyr = Sxy[xp + iy * nx];
                T Sxyl = Sxy[xm + iy * nx], Sxytl = Sxy[xm + yp * nx];
                Fx[i] = -1 * (Sxxr - Sxxi) / dxf - 0.5f * (Sxyt + Sxytr - Sxyb - Sxybr) / (2.0f * dxf);
                Fy[i] = -1 * (Syyt - Syyi) / dxf - 0.5f * (Sxyr + Sxytr - Sxyl - Sxytl) / (2.0f * dxf);
            }
        twodimbnd(Fx, false);
        twodimbnd(Fy, true);
        /* breakerdelayCPU (wave_CPU.cpp:1333-1368) */
        T* urms = f(XBG_F_URMS); T* ust = f(XBG_F_UST);
        for (int i = 0; i < C; i++) {
            T hmin = (T)0.2;
            T Hi = H[i], ki = k[i];
            T hhi = cmax(hh[i], hmin);
            T ci = cmax(c[i], M<T>::sqrt(hmin * g));
            T Rl = R[i];
            T uorb = (T)(REF_PI * Hi / Trep / M<T>::sinh(cmin(cmax(ki, (T)0.01f) * hhi, (T)10.0f)));
            urms[i] = uorb / (M<T>::sqrt((T)2.0f));
            T ustw = E[i] / ci / rho / hhi;
            T ustr = 2.0f * Rl / ci / rho / hhi;
            ust[i] = ustw + ustr;
        }
        twodimbnd(ust, true);
        return XBG_OK;
    }

    /* ========================================================= flow step */
    static inline T minmod(T d1, T d2) {   /* Flow_kernel.cu:23-41 */
        T r = 0.0f;
        if (d1 * d2 > 0.0f) {
            if (d1 > 0.0f) r = M<T>::fmin(d1, d2);
            if (d1 < 0.0f) r = M<T>::fmax(d1, d2);
        }
        return r;
    }
    /* latbnd (Flow_kernel.cu:1778-1809): rows 0/ny-1 <- rows 1/ny-2 */
    void latbnd(T* q) {
        for (int ix = 0; ix < nx; ix++) {
            T a = q[ix + 1 * nx], b = q[ix + (ny - 2) * nx];
            q[ix] = a; q[ix + (ny - 1) * nx] = b;
        }
    }
    /* zblatbnd (Sediment_kernel.cu:970-1018) */
    void zblatbnd(T* q) {
        std::vector<T> o(q, q + C);
        for (int iy = 0; iy < ny; iy++)
            for (int ix = 0; ix < nx; ix++) {
                int i = ix + iy * nx;
                if (iy == 0) q[i] = o[ix + pp(iy, ny) * nx];
                if (iy == ny - 1) q[i] = o[ix + mm(iy) * nx];
                if (ix == 0) q[i] = o[pp(ix, nx) + iy * nx];
            }
    }

    int flow_step() override {   /* flowstep, Wave_gpu.cu:1106-1403 */
        if (status != XBG_OK) return status;
        T* zs = f(XBG_F_ZS); T* zb = f(XBG_F_ZB); T* hh = f(XBG_F_HH);
        T* uu = f(XBG_F_UU); T* vv = f(XBG_F_VV); T* hu = f(XBG_F_HU);
        T* hv = f(XBG_F_HV); T* hum = f(XBG_F_HUM); T* hvm = f(XBG_F_HVM);
        T* qx = f(XBG_F_QX); T* qy = f(XBG_F_QY);
        T* uuold = f(XBG_F_UUOLD); T* vvold = f(XBG_F_VVOLD); T* zsold = f(XBG_F_ZSOLD);
        T* DR = f(XBG_F_DR); T* cfm = f(XBG_F_CFM); T* urms = f(XBG_F_URMS);
        T* Fx = f(XBG_F_FX); T* Fy = f(XBG_F_FY);
        T* vu = f(XBG_F_VU); T* uv = f(XBG_F_UV); T* ueu = f(XBG_F_UEU); T* vev = f(XBG_F_VEV);
        T* vmageu = f(XBG_F_VMAGEU); T* vmagev = f(XBG_F_VMAGEV);
        T* dzsdt = f(XBG_F_DZSDT);
        T dx = (T)P.dx, dtf = (T)dt, eps = (T)P.eps, g = (T)P.g, rho = (T)P.rho;
        T nuhfac = (T)P.nuhfac, nuh = (T)P.nuh;
        const T ummn = 0.0f;   /* uumin, Wave_gpu.cu:65 */
        auto I = [&](int x, int y) { return x + y * nx; };
        /* wlevslopes (Flow_kernel.cu:410-465) */
        for (int iy = 0; iy < ny; iy++)
            for (int ix = 0; ix < nx; ix++) {
                int i = I(ix, iy);
                dzsdx[i] = (zs[I(pp(ix, nx), iy)] - zs[i]) / dx;
                dzsdy[i] = (zs[I(ix, pp(iy, ny))] - zs[i]) / dx;
            }
        /* udepthmomcont / vdepthmomcont (:546-651) */
        for (int iy = 0; iy < ny; iy++)
            for (int ix = 0; ix < nx; ix++) {
                int i = I(ix, iy);
                T humi = 0.5f * (hh[i] + hh[I(pp(ix, nx), iy)]);
                wetu[i] = (hu[i] > eps && humi > eps) ? 1 : 0;
                hum[i] = M<T>::fmax(humi, eps);
                T hvmi = 0.5f * (hh[i] + hh[I(ix, pp(iy, ny))]);
                wetv[i] = (hv[i] > eps && hvmi > eps) ? 1 : 0;
                hvm[i] = M<T>::fmax(hvmi, eps);
            }
        /* ududx_adv (:752-824), vdudy_adv (:887-949) */
        for (int iy = 0; iy < ny; iy++)
            for (int ix = 0; ix < nx; ix++) {
                int i = I(ix, iy);
                int xm = mm(ix), xp = pp(ix, nx), ym = mm(iy), yp = pp(iy, ny);
                T uui = uu[i], uur = uu[I(xp, iy)], uul = uu[I(xm, iy)];
                T r = 0.0f;
                T qin = 0.5f * (hu[i] * uui + hu[I(xm, iy)] * uul);
                T du = uui - uul;
                if (qin > 0.0f) {
                    if (du > 0.5f) r = r + 0.5f * (uul + uui) * (uui - uul) / dx;
                    else r = r + qin / hum[i] * (uui - uul) / dx;
                }
                qin = -0.5f * (hu[i] * uui + hu[I(xp, iy)] * uur);
                du = uur - uui;
                if (qin > 0.0f) {
                    if (du > 0.5f) r = r - 0.5f * (uur + uui) * (uui - uur) / dx;
                    else r = r + qin / hum[i] * (uui - uur) / dx;
                }
                ududx[i] = r;
                T uut = uu[I(ix, yp)], uub = uu[I(ix, ym)];
                T s = 0.0f;
                qin = 0.5f * (vv[I(ix, ym)] * hv[I(ix, ym)] + vv[I(xp, ym)] * hv[I(xp, ym)]);
                T dv = vv[i] - vv[I(ix, ym)];
                if (qin > 0.0f) {
                    if (dv > 0.5f) s = s + 0.5f * (vv[I(ix, ym)] + vv[I(xp, ym)]) * (uui - uub) / dx;
                    else s = s + qin / hum[i] * (uui - uub) / dx;
                }
                qin = -0.5f * (vv[i] * hv[i] + vv[I(xp, iy)] * hv[I(xp, iy)]);
                dv = vv[I(ix, yp)] - vv[i];
                if (qin > 0.0f) {
                    if (dv > 0.5f) s = s - 0.5f * (vv[i] + vv[I(xp, iy)]) * (uui - uut) / dx;
                    else s = s + qin / hum[i] * (uui - uut) / dx;
                }
                vdudy[i] = s;
            }
        /* smago (:1282-1316) */
        for (int iy = 0; iy < ny; iy++)
            for (int ix = 0; ix < nx; ix++) {
                int i = I(ix, iy);
                int xm = mm(ix), xp = pp(ix, nx), ym = mm(iy), yp = pp(iy, ny);
                if (P.usesmago == 1) {
                    T dudx = (uu[i] - uu[I(xm, iy)]) / dx;
                    T dudy = 0.50f * (uu[I(ix, yp)] - uu[I(ix, ym)] + uu[I(xm, yp)] - uu[I(xm, ym)]) / dx;
                    T dvdy = (vv[i] - vv[I(ix, ym)]) / dx;
                    T dvdx = 0.50f * (vv[I(xp, iy)] - vv[I(xm, iy)] + vv[I(xp, ym)] - vv[I(xm, ym)]) / dx;
                    T tau = M<T>::sqrt(2.0f * dudx * dudx + 2.0f * dvdy * dvdy + M<T>::pow(dudy + dvdx, 2.0f));
                    nuhg[i] = M<T>::fmax(nuh * nuh * dx * dx * tau, nuhfac * hh[i] * M<T>::pow(DR[i] / rho, 1.0f / 3.0f));
                } else {
                    nuhg[i] = M<T>::fmax(nuh, nuhfac * hh[i] * M<T>::pow(DR[i] / rho, 1.0f / 3.0f));
                }
            }
        /* viscou1 + viscou2 (:1319-1396) */
        for (int iy = 0; iy < ny; iy++)
            for (int ix = 0; ix < nx; ix++) {
                int i = I(ix, iy);
                int xm = mm(ix), xp = pp(ix, nx), ym = mm(iy), yp = pp(iy, ny);
                T nuh1 = nuhg[I(xp, iy)], nuh2 = nuhg[i];
                T dudx1 = nuh1 * hh[I(xp, iy)] * (uu[I(xp, iy)] - uu[i]) / dx;
                T dudx2 = nuh2 * hh[i] * (uu[i] - uu[I(xm, iy)]) / dx;
                T v = (1.0f / hum[i]) * ((dudx1 - dudx2) / (dx));
                nuh1 = 0.25f * (nuhg[i] + nuhg[I(xp, iy)] + nuhg[I(xp, yp)] + nuhg[I(ix, yp)]);
                nuh2 = 0.25f * (nuhg[i] + nuhg[I(xp, iy)] + nuhg[I(xp, ym)] + nuhg[I(ix, ym)]);
                T dudy1 = nuh1 * 0.5f * (hvm[i] + hvm[I(xp, iy)]) * (uu[I(ix, yp)] - uu[i]) / dx;
                T dudy2 = nuh2 * 0.5f * (hvm[I(ix, ym)] + hvm[I(xp, ym)]) * (uu[i] - uu[I(ix, ym)]) / dx;
                viscu[i] = v + (1.0f / hum[i]) * ((dudy1 - dudy2) / dx * wetu[I(ix, yp)] * wetu[I(ix, ym)]);
            }
        /* eulerustep (:1487-1544) */
        T fc = (T)P.fc, Cd = (T)P.Cd, wu = (T)windu, wv = (T)windv;
        {
            std::vector<T> nu(uu, uu + C);
            int sw = (wu > 0.0) - (wu < 0.0);
            for (int iy = 0; iy < ny; iy++)
                for (int ix = 0; ix < nx; ix++) {
                    int i = I(ix, iy);
                    T hmin = (T)0.2;
                    T uui = uu[i];
                    if (wetu[i] == 1) {
                        T taubx = cfm[i] * rho * ueu[i] * M<T>::sqrt(1.3456f * urms[i] * urms[i] + vmageu[i] * vmageu[i]);
                        uui = uui - dtf * (ududx[i] + vdudy[i] - viscu[i] + g * dzsdx[i] + taubx / (rho * hu[i]) -
                                           Fx[i] / (rho * M<T>::fmax(hum[i], hmin)) -
                                           1.25f * Cd * sw * wu * wu / (rho * hum[i]) - fc * vu[i]);
                    } else {
                        uui = 0.0f;
                    }
                    if (ix > 0) nu[i] = uui;
                }
            std::copy(nu.begin(), nu.end(), uu);
        }
        latbnd(uu);
        /* vdvdy_adv (:1024-1074) + vdvdy_fixbnd at iy = ny-1 (deviation 2) */
        for (int iy = 0; iy < ny; iy++)
            for (int ix = 0; ix < nx; ix++) {
                int i = I(ix, iy);
                int ym = mm(iy), yp = pp(iy, ny);
                T r = 0.0f;
                if (ix > 0 && iy > 0 && iy < (ny - 2)) {
                    T qin = 0.5f * (vv[i] * hv[i] + vv[I(ix, ym)] * hv[I(ix, ym)]);
                    T dv = vv[i] - vv[I(ix, ym)];
                    if (qin > 0.0f) {
                        if (dv > 0.5f) r = r + 0.5f * (vv[I(ix, ym)] - vv[i]) * (vv[i] - vv[I(ix, ym)]) / (dx);
                        else r = r + qin / hvm[i] * (vv[i] - vv[I(ix, ym)]) / (dx);
                    }
                    qin = -0.5f * (hv[i] * vv[i] + hv[I(ix, yp)] * vv[I(ix, yp)]);
                    dv = vv[I(ix, yp)] - vv[i];
                    if (qin > 0.0f) {
                        if (dv > 0.5f) r = r - 0.5f * (vv[I(ix, yp)] + vv[i]) * (vv[i] - vv[I(ix, yp)]) / (dx);
                        else r = r + qin / hvm[i] * (vv[i] - vv[I(ix, yp)]) / (dx);
                    }
                }
                if (ix > 0 && iy > 0 && iy == ny - 1) {
                    T qin = 0.5f * (vv[i] * hv[i] + vv[I(ix, ym)] * hv[I(ix, ym)]);
                    if (qin > 0.0f) r = r + qin / hvm[i] * (vv[i] - vv[I(ix, ym)]) / (dx);
                }
                vdvdy[i] = r;
            }
        /* udvdx_adv (:1159-1210), with the updated uu */
        for (int iy = 0; iy < ny; iy++)
            for (int ix = 0; ix < nx; ix++) {
                int i = I(ix, iy);
                int xm = mm(ix), xp = pp(ix, nx), yp = pp(iy, ny);
                T r = 0.0f;
                T qin = (T)(0.5 * (uu[I(xm, iy)] * hu[I(xm, iy)] + uu[I(xm, yp)] * hu[I(xm, yp)]));
                T du = uu[i] - uu[I(xm, iy)];
                if (qin > 0.0f) {
                    if (du > 0.5f) r = r + 0.5f * (uu[I(xm, iy)] + uu[I(xm, yp)]) * (vv[i] - vv[I(xm, iy)]) / (dx);
                    else r = r + qin / hvm[i] * (vv[i] - vv[I(xm, iy)]) / (dx);
                }
                qin = (T)(-0.5 * (uu[i] * hu[i] + uu[I(ix, yp)] * hu[I(ix, yp)]));
                du = uu[I(xp, iy)] - uu[i];
                if (qin > 0.0f) {
                    if (du > 0.5f) r = r - 0.5f * (uu[i] + uu[I(xp, iy)]) * (vv[i] - vv[I(xp, iy)]) / (dx);
                    else r = r + qin / hvm[i] * (vv[i] - vv[I(xp, iy)]) / (dx);
                }
                udvdx[i] = r;
            }
        /* viscov1 (:1399-1428), viscovbnd (:1461-1484), viscov2 (:1430-1459) */
        for (int iy = 0; iy < ny; iy++)
            for (int ix = 0; ix < nx; ix++) {
                int i = I(ix, iy);
                int ym = mm(iy), yp = pp(iy, ny);
                T nuh1 = nuhg[I(ix, yp)], nuh2 = nuhg[i];
                T dvdy1 = nuh1 * hh[I(ix, yp)] * (vv[I(ix, yp)] - vv[i]) / dx;
                T dvdy2 = nuh2 * hh[i] * (vv[i] - vv[I(ix, ym)]) / dx;
                viscv[i] = (1.0f / hvm[i]) * (dvdy1 - dvdy2) / dx * wetv[I(ix, yp)] * wetv[I(ix, ym)];
            }
        for (int ix = 0; ix < nx; ix++) {
            T a = viscv[I(ix, mm(ny - 2))], b = viscv[I(ix, pp(0, ny))];
            viscv[I(ix, ny - 2)] = a;
            viscv[I(ix, 0)] = b;
        }
        for (int iy = 0; iy < ny; iy++)
            for (int ix = 0; ix < nx; ix++) {
                int i = I(ix, iy);
                int xm = mm(ix), xp = pp(ix, nx), yp = pp(iy, ny);
                T nuh1 = 0.25f * (nuhg[i] + nuhg[I(xp, iy)] + nuhg[I(xp, yp)] + nuhg[I(ix, yp)]);
                T nuh2 = 0.25f * (nuhg[i] + nuhg[I(xm, iy)] + nuhg[I(xm, yp)] + nuhg[I(ix, yp)]);
                T dvdx1 = nuh1 * 0.5f * (hum[i] + hum[I(ix, yp)]) * (vv[I(xp, iy)] - vv[i]) / dx;
                T dvdx2 = nuh2 * 0.5f * (hum[I(xm, iy)] + hum[I(xm, yp)]) * (vv[i] - vv[I(xm, iy)]) / dx;
                viscv[i] = viscv[i] + (1.0f / hvm[i]) * ((dvdx1 - dvdx2) / (dx) * wetv[I(xp, iy)] * wetv[I(xm, iy)]);
            }
        /* eulervstep (:1546-1599) */
        {
            int sw = (wv > 0.0) - (wv < 0.0);
            for (int iy = 0; iy < ny - 2; iy++)
                for (int ix = 0; ix < nx; ix++) {
                    int i = I(ix, iy);
                    T hmin = (T)0.2;
                    T vvi = vv[i];
                    if (wetv[i] == 1) {
                        T tauby = cfm[i] * rho * vev[i] * M<T>::sqrt(1.3456f * urms[i] * urms[i] + vmagev[i] * vmagev[i]);
                        vvi = vvi - dtf * (udvdx[i] + vdvdy[i] - viscv[i] + g * dzsdy[i] + tauby / (rho * hv[i]) -
                                           Fy[i] / (rho * M<T>::fmax(hvm[i], hmin)) + fc * uv[i] -
                                           1.25f * Cd * sw * wv * wv / (rho * hvm[i]));
                    } else {
                        vvi = 0.0f;
                    }
                    if (ix > 0) vv[i] = vvi;
                }
        }
        /* vvlatbnd (:1812-1846) */
        for (int ix = 0; ix < nx; ix++) {
            T a = vv[I(ix, pp(0, ny))], b = vv[I(ix, mm(ny - 2))];
            vv[I(ix, 0)] = a; vv[I(ix, ny - 2)] = b;
        }
        /* wrkuu2Ocorr (:1960-2044) + uu2Ocorr (:2210-2245) */
        for (int iy = 0; iy < ny; iy++)
            for (int ix = 0; ix < nx; ix++) {
                int i = I(ix, iy);
                int xm = mm(ix), xm2 = mm2(ix), xp = pp(ix, nx), xp2 = pp2(ix, nx);
                int ym = mm(iy), yp = pp(iy, ny), yp2 = pp2(iy, ny);
                T w1 = 0.0f, w2 = 0.0f;
                T minzs = M<T>::fmin(M<T>::fmin(M<T>::fmin(M<T>::fmin(zs[I(xm2, iy)], zs[I(xm, iy)]), zs[i]), zs[I(xp, iy)]), zs[I(xp2, iy)]);
                T minzb = M<T>::fmin(M<T>::fmin(M<T>::fmin(M<T>::fmin(zb[I(xm2, iy)], zb[I(xm, iy)]), zb[i]), zb[I(xp, iy)]), zb[I(xp2, iy)]);
                T mindepth = minzs + minzb;
                if (ix > 0 && mindepth > eps * 2.0f) {
                    if ((qx[i] + qx[I(xm, iy)]) > 0.0f)
                        w1 = 0.5f * minmod(uu[i] - uuold[I(xm, iy)], uu[I(xm, iy)] - uuold[I(xm2, iy)]);
                    if ((qx[i] + qx[I(xm, iy)]) < 0.0f)
                        w1 = -0.5f * minmod(uuold[i] - uu[I(xm, iy)], uuold[I(xp, iy)] - uu[i]);
                }
                minzs = M<T>::fmin(M<T>::fmin(M<T>::fmin(zs[I(ix, iy)], zs[I(ix, ym)]), zs[I(ix, yp)]), zs[I(ix, yp2)]);
                minzs = M<T>::fmin(minzs, M<T>::fmin(M<T>::fmin(M<T>::fmin(zs[I(xp, iy)], zs[I(xp, ym)]), zs[I(xp, yp)]), zs[I(xp, yp2)]));
                minzb = M<T>::fmin(M<T>::fmin(M<T>::fmin(zb[I(ix, iy)], zb[I(ix, ym)]), zb[I(ix, yp)]), zb[I(ix, yp2)]);
                minzb = M<T>::fmin(minzb, M<T>::fmin(M<T>::fmin(M<T>::fmin(zb[I(xp, iy)], zb[I(xp, ym)]), zb[I(xp, yp)]), zb[I(xp, yp2)]));
                mindepth = minzs + minzb;
                if (ix > 0 && iy > 0 && mindepth > eps * 2.0f) {
                    if ((qy[I(xp, iy)] + qy[i]) > 0.0f)
                        w2 = 0.5f * minmod(uu[I(ix, yp)] - uuold[i], uu[i] - uuold[I(ix, ym)]);
                    if ((qy[I(xp, iy)] + qy[i]) < 0.0f)
                        w2 = -0.5f * minmod(uuold[I(ix, yp)] - uu[i], uuold[I(ix, yp2)] - uu[I(ix, yp)]);
                }
                wrk1[i] = w1; wrk2[i] = w2;
            }
        {
            std::vector<T> nu(uu, uu + C);
            for (int iy = 1; iy < ny; iy++)
                for (int ix = 1; ix < nx; ix++) {
                    int i = I(ix, iy);
                    int xm = mm(ix), xp = pp(ix, nx), ym = mm(iy);
                    T qe = 0.5f * (qx[I(xp, iy)] + qx[i]);
                    T qw = 0.5f * (qx[i] + qx[I(xm, iy)]);
                    T qn = 0.5f * (qy[I(ix, ym)] + qy[I(xp, ym)]);
                    T qs = 0.5f * (qy[i] + qy[I(xm, iy)]);
                    nu[i] = uu[i] - dtf / hum[i] * ((qe * wrk1[I(xp, iy)] - qw * wrk1[i]) / dx + (qs * wrk2[i] - qn * wrk2[I(ix, ym)]) / dx);
                }
            std::copy(nu.begin(), nu.end(), uu);
        }
        /* wrkvv2Ocorr (:2046-2128) + vv2Ocorr (:2247-2282) */
        for (int iy = 0; iy < ny; iy++)
            for (int ix = 0; ix < nx; ix++) {
                int i = I(ix, iy);
                int xm = mm(ix), xp = pp(ix, nx), xp2 = pp2(ix, nx);
                int ym = mm(iy), ym2 = mm2(iy), yp = pp(iy, ny), yp2 = pp2(iy, ny);
                T w1 = 0.0f, w2 = 0.0f;
                T minzs = M<T>::fmin(M<T>::fmin(M<T>::fmin(M<T>::fmin(zs[I(ix, ym2)], zs[I(ix, ym)]), zs[I(ix, iy)]), zs[I(ix, yp)]), zs[I(ix, yp2)]);
                T minzb = M<T>::fmin(M<T>::fmin(M<T>::fmin(M<T>::fmin(zb[I(ix, ym2)], zb[I(ix, ym)]), zb[I(ix, iy)]), zb[I(ix, yp)]), zb[I(ix, yp2)]);
                T mindepth = minzs + minzb;
                if (ix > 0 && iy > 0 && iy < ny - 2 && mindepth > eps * 2.0f) {
                    if ((qy[i] + qy[I(ix, ym)]) > 0.0f)
                        w1 = 0.5f * minmod(vv[i] - vvold[I(ix, ym)], vv[I(ix, ym)] - vvold[I(ix, ym2)]);
                    if ((qy[i] + qy[I(ix, ym)]) < 0.0f)
                        w1 = -0.5f * minmod(vvold[i] - vv[I(ix, ym)], vvold[I(ix, yp)] - vv[i]);
                }
                minzs = M<T>::fmin(M<T>::fmin(M<T>::fmin(zs[I(xm, iy)], zs[I(ix, iy)]), zs[I(xp, iy)]), zs[I(xp2, iy)]);
                minzs = M<T>::fmin(minzs, M<T>::fmin(M<T>::fmin(M<T>::fmin(zs[I(xm, yp)], zs[I(ix, yp)]), zs[I(xp, yp)]), zs[I(xp2, yp)]));
                minzb = M<T>::fmin(M<T>::fmin(M<T>::fmin(zb[I(xm, iy)], zb[I(ix, iy)]), zb[I(xp, iy)]), zb[I(xp2, iy)]);
                minzb = M<T>::fmin(minzb, M<T>::fmin(M<T>::fmin(M<T>::fmin(zb[I(xm, yp)], zb[I(ix, yp)]), zb[I(xp, yp)]), zb[I(xp2, yp)]));
                mindepth = minzs + minzb;
                if (ix > 0 && iy > 0 && iy < ny - 2 && mindepth > eps * 2.0f) {
                    if ((qx[I(ix, yp)] + qx[i]) > 0.0f)
                        w2 = 0.5f * minmod(vv[I(xp, iy)] - vvold[i], vv[i] - vvold[I(xm, iy)]);
                    if ((qx[I(ix, yp)] + qx[i]) < 0.0f)
                        w2 = -0.5f * minmod(vvold[I(xp, iy)] - vv[i], vvold[I(xp2, iy)] - vv[I(xp, iy)]);
                }
                wrk1[i] = w1; wrk2[i] = w2;
            }
        {
            std::vector<T> nv(vv, vv + C);
            for (int iy = 1; iy < ny; iy++)
                for (int ix = 1; ix < nx; ix++) {
                    int i = I(ix, iy);
                    int xm = mm(ix), ym = mm(iy), yp = pp(iy, ny);
                    T qe = 0.5f * (qx[I(ix, yp)] + qx[i]);
                    T qw = 0.5f * (qx[I(xm, iy)] + qx[I(xm, yp)]);
                    T qn = 0.5f * (qy[i] + qy[I(ix, ym)]);
                    T qs = 0.5f * (qy[I(ix, yp)] + qy[i]);
                    nv[i] = vv[i] - dtf / hvm[i] * ((qe * wrk2[i] - qw * wrk2[I(xm, iy)]) / dx + (qs * wrk1[I(ix, yp)] - qn * wrk1[i]) / dx);
                }
            std::copy(nv.begin(), nv.end(), vv);
        }
        /* depthhu / depthhv (:653-750) */
        for (int iy = 0; iy < ny; iy++)
            for (int ix = 0; ix < nx; ix++) {
                int i = I(ix, iy);
                int xp = pp(ix, nx), yp = pp(iy, ny);
                T h;
                T bu = M<T>::fmax(-1.0f * zb[i], -1.0f * zb[I(xp, iy)]);
                if (uu[i] > ummn) h = zs[i] - bu;
                else if (uu[i] < -1.0f * ummn) h = zs[I(xp, iy)] - bu;
                else h = M<T>::fmax(M<T>::fmax(zs[i], zs[I(xp, iy)]) - bu, eps);
                hu[i] = M<T>::fmax(h, 0.0f);
                T bv = M<T>::fmax(-1.0f * zb[i], -1.0f * zb[I(ix, yp)]);
                if (vv[i] > ummn) h = zs[i] - bv;
                else if (vv[i] < -1 * ummn) h = zs[I(ix, yp)] - bv;
                else h = M<T>::fmax(M<T>::fmax(zs[i], zs[I(ix, yp)]) - bv, eps);
                hv[i] = M<T>::fmax(h, 0.0f);
            }
        /* CalcQFlow (:1917-1958) */
        for (int i = 0; i < C; i++) { qx[i] = uu[i] * hu[i]; qy[i] = vv[i] * hv[i]; }
        /* continuity (:1626-1681) */
        {
            std::vector<T> nz(zs, zs + C);
            for (int iy = 0; iy < ny; iy++)
                for (int ix = 1; ix < nx; ix++) {
                    int i = I(ix, iy);
                    T dzdt = (qx[I(mm(ix), iy)] - qx[i] + qy[I(ix, mm(iy))] - qy[i]) / dx;
                    dzsdt[i] = dzdt;
                    nz[i] = zs[i] + dzdt * dtf;
                }
            std::copy(nz.begin(), nz.end(), zs);
        }
        /* wrkzs2Ocorr (:2130-2208) + zs2Ocorr (:2284-2317) */
        for (int iy = 0; iy < ny; iy++)
            for (int ix = 0; ix < nx; ix++) {
                int i = I(ix, iy);
                int xm = mm(ix), xp = pp(ix, nx), xp2 = pp2(ix, nx);
                int ym = mm(iy), yp = pp(iy, ny), yp2 = pp2(iy, ny);
                T w1 = 0.0f, w2 = 0.0f;
                T minzs = M<T>::fmin(M<T>::fmin(M<T>::fmin(zs[I(xm, iy)], zs[i]), zs[I(xp, iy)]), zs[I(xp2, iy)]);
                T minzb = M<T>::fmin(M<T>::fmin(M<T>::fmin(zb[I(xm, iy)], zb[i]), zb[I(xp, iy)]), zb[I(xp2, iy)]);
                T mindepth = minzs + minzb;
                if (ix > 0 && mindepth > eps * 2.0f) {
                    if ((uu[i]) > 0.0f)
                        w1 = uu[i] * 0.5f * minmod(zs[I(xp, iy)] - zsold[i], zs[i] - zsold[I(xm, iy)]);
                    if ((uu[i]) < 0.0f)
                        w1 = -1.0f * uu[i] * 0.5f * minmod(zsold[I(xp2, iy)] - zs[I(xp, iy)], zsold[I(xp, iy)] - zs[i]);
                }
                minzs = M<T>::fmin(M<T>::fmin(M<T>::fmin(zs[I(ix, ym)], zs[i]), zs[I(ix, yp)]), zs[I(ix, yp2)]);
                minzb = M<T>::fmin(M<T>::fmin(M<T>::fmin(zb[I(ix, ym)], zb[i]), zb[I(ix, yp)]), zb[I(ix, yp2)]);
                mindepth = minzs + minzb;
                if (ix > 0 && iy > 0 && mindepth > eps * 2.0f) {
                    if ((vv[i]) > 0.0f)
                        w2 = vv[i] * 0.5f * minmod(zs[I(ix, yp)] - zsold[i], zs[i] - zsold[I(ix, ym)]);
                    if ((vv[i]) < 0.0f)
                        w2 = vv[i] * 0.5f * minmod(zsold[I(ix, yp2)] - zs[I(ix, yp)], zsold[I(ix, yp)] - zs[i]);
                }
                wrk1[i] = w1; wrk2[i] = w2;
            }
        {
            std::vector<T> nz(zs, zs + C);
            for (int iy = 1; iy < ny; iy++)
                for (int ix = 1; ix < nx; ix++) {
                    int i = I(ix, iy);
                    nz[i] = zs[i] - dtf * ((wrk1[i] - wrk1[I(mm(ix), iy)]) / dx + (wrk2[i] - wrk2[I(ix, mm(iy))]) / dx);
                    qx[i] = qx[i] + wrk1[i];
                    qy[i] = qy[i] + wrk2[i];
                }
            std::copy(nz.begin(), nz.end(), zs);
        }
        latbnd(zs);
        /* hsbnd (:1683-1710) */
        for (int i = 0; i < C; i++) hh[i] = M<T>::fmax(zb[i] + zs[i], eps);
        /* calcuvvu (:467-544) */
        const T* ust = f(XBG_F_UST); const T* thm = f(XBG_F_THETAMEAN);
        for (int iy = 0; iy < ny; iy++)
            for (int ix = 0; ix < nx; ix++) {
                int i = I(ix, iy);
                int xm = mm(ix), xp = pp(ix, nx), ym = mm(iy), yp = pp(iy, ny);
                T usti = ust[i], tmi = thm[i];
                T ustr = ust[I(xp, iy)], tmr = thm[I(xp, iy)];
                T ustt = ust[I(ix, yp)], tmt = thm[I(ix, yp)];
                T wu_ = (T)wetu[i], wv_ = (T)wetv[i];
                uuold[i] = uu[i]; vvold[i] = vv[i]; zsold[i] = zs[i];
                vu[i] = 0.25f * (vv[I(ix, ym)] + vv[I(ix, iy)] + vv[I(xp, ym)] + vv[I(xp, iy)]) * wu_;
                uv[i] = 0.25f * (uu[I(xm, iy)] + uu[I(ix, iy)] + uu[I(xm, yp)] + uu[I(ix, yp)]) * wv_;
                T vsu = 0.5f * (usti * M<T>::sin(tmi) + ustr * M<T>::sin(tmr)) * wu_;
                T usu = 0.5f * (usti * M<T>::cos(tmi) + ustr * M<T>::cos(tmr)) * wu_;
                T ue = uu[i] - usu;
                T ve = vu[i] - vsu;
                vmageu[i] = M<T>::sqrt(ue * ue + ve * ve);
                ueu[i] = ue;
                T usv = 0.5f * (usti * M<T>::cos(tmi) + ustt * M<T>::cos(tmt)) * wv_;
                T vsv = 0.5f * (usti * M<T>::sin(tmi) + ustt * M<T>::sin(tmt)) * wv_;
                T vvv = vv[i] - vsv;
                T uvv = uv[i] - usv;
                vmagev[i] = M<T>::sqrt(uvv * uvv + vvv * vvv);
                vev[i] = vvv;
            }
        /* uvlatbnd (:1712-1776) */
        latbnd(uv); latbnd(vu); latbnd(ueu); latbnd(vev); latbnd(vmageu); latbnd(vmagev);
        return XBG_OK;
    }

    /* ====================================================== sediment step */
    void updatezom() {   /* Sediment_kernel.cu:1162-1190 */
        const T* st = f(XBG_F_STDEP);
        T* cfm = f(XBG_F_CFM); T* fwm = f(XBG_F_FWM);
        for (int i = 0; i < C; i++) {
            if (st[i] < 0.05f) { cfm[i] = (T)P.cfreef; fwm[i] = (T)P.fwreef; }
            else { cfm[i] = (T)P.cfsand; fwm[i] = (T)P.fwsand; }
        }
    }

    int sediment_step() override {   /* sedimentstep, Wave_gpu.cu:1405-1635 */
        if (status != XBG_OK) return status;
        if (!(P.sedtrans == 1 && totaltime >= P.sedstart)) return XBG_OK;
        T* hh = f(XBG_F_HH); T* zb = f(XBG_F_ZB); T* zs = f(XBG_F_ZS);
        T* uu = f(XBG_F_UU); T* vv = f(XBG_F_VV);
        T* c = f(XBG_F_C); T* dzsdt = f(XBG_F_DZSDT);
        T* rolthick = f(XBG_F_ROLTHICK); T* kturb = f(XBG_F_KTURB);
        T* ueu = f(XBG_F_UEU); T* vev = f(XBG_F_VEV);
        T* H = f(XBG_F_H); T* DR = f(XBG_F_DR); T* R = f(XBG_F_R);
        T* urms = f(XBG_F_URMS); T* ceqsg = f(XBG_F_CEQSG); T* cfm = f(XBG_F_CFM);
        T* stdep = f(XBG_F_STDEP); T* Cc = f(XBG_F_CC); T* dzb = f(XBG_F_DZB);
        T* hu = f(XBG_F_HU); T* hv = f(XBG_F_HV); T* uvg = f(XBG_F_UV); T* vug = f(XBG_F_VU);
        T* thm = f(XBG_F_THETAMEAN);
        T dx = (T)P.dx, dtf = (T)dt, eps = (T)P.eps, g = (T)P.g, rho = (T)P.rho;
        T nuhfac = (T)P.nuhfac, nuh = (T)P.nuh, beta = (T)P.beta;
        auto I = [&](int x, int y) { return x + y * nx; };
        /* longturb (Sediment_kernel.cu:27-164): rolthick, kturb = 0 */
        for (int i = 0; i < C; i++) {
            T dzsdt_cr = beta * c[i];
            T rolth = rolthick[i] + dtf * (M<T>::fabs(dzsdt[i]) - dzsdt_cr);
            rolthick[i] = M<T>::fmax(rolth, 0.0f);
        }
        /* Sbvr (:167-326) reads kturb before longturb zeroes it?  No:
           longturb runs first and sets kturb = 0 for every cell. */
        for (int i = 0; i < C; i++) kturb[i] = 0.0f;
        T D50 = (T)P.D50, D90 = (T)P.D90, rhosed = (T)P.rhosed, ws = (T)P.wws;
        for (int iy = 0; iy < ny; iy++)
            for (int ix = 0; ix < nx; ix++) {
                int i = I(ix, iy);
                int xm = mm(ix), ym = mm(iy);
                T zo = 0.006f, sedcal = 1.0f, bulk = 1.0f;
                T drho = (rhosed - rho) / rho;
                T dester = M<T>::pow(drho * g, 1.0f / 3.0f) / 0.0001f * D50;
                T hhi = M<T>::fmax(hh[i], 0.01f);
                T ue = (T)(0.5 * (ueu[I(xm, iy)] + ueu[i]));
                T ve = (T)(0.5 * (vev[I(ix, ym)] + vev[i]));
                T vmags = ue * ue + ve * ve;
                T ML = M<T>::fmax(M<T>::fmin(M<T>::sqrt(2.0f * R[i] * Trep / (rho * c[i])), hhi), 0.01f);
                T dcfin = M<T>::exp(M<T>::fmin(hhi, 100.0f) / ML);
                T dcf = M<T>::fmin(1 / (dcfin - 1), 1.0f);
                T kb = nuhfac * M<T>::pow(DR[i] / rho, 0.66666666667f) * dcf;
                T Urms2 = urms[i] * urms[i] + 1.45f * (kb + kturb[i]);
                T tsfac = 0.1f, Tsmin = 0.5f;
                Tsg[i] = M<T>::fmax(tsfac * hhi / ws, Tsmin);
                T Ucr;
                if (D50 <= 0.0005f) Ucr = 0.19f * M<T>::pow(D50, 0.1f) * M<T>::log10(4.0f * hhi / D90);
                else Ucr = 8.50f * M<T>::pow(D50, 0.6f) * M<T>::log10(4.0f * hhi / D90);
                T hdrag = M<T>::fmax(hhi, 10.0f * zo);
                T Cd = 0.4f / (M<T>::log(hdrag / zo) - 1.0f);
                Cd = Cd * Cd;
                T Asb = 0.005f * hhi * M<T>::pow(1 / hhi / (drho * g), 1.2f);
                T Ass = 0.012f * D50 * M<T>::pow(dester, -0.6f) / (M<T>::pow(drho * g * D50, 1.2f));
                T T1 = vmags + 0.018f / Cd * Urms2;
                T1 = M<T>::fmin(T1, 100000.0f * g / cfm[i] * D50 * drho);
                T1 = M<T>::sqrt(T1);
                int wetz = hhi > eps ? 1 : 0;
                T T2 = 0.0f;
                if (T1 > Ucr && hhi > eps) T2 = M<T>::pow(T1 - Ucr, 2.4f);
                T ceqb = Asb * T2;
                ceqb = M<T>::fmin(ceqb / hhi, 0.05f);
                ceqbg[i] = (1 - bulk) * ceqb * sedcal * wetz;
                T ceqs = M<T>::fmin(Ass * T2 / hhi, 0.05f);
                ceqsg[i] = (ceqs + bulk * ceqb) * sedcal * wetz;
            }
        /* Rvr (:477-509) */
        T facsk = (T)P.facsk, facas = (T)P.facas;
        for (int i = 0; i < C; i++) {
            T m1 = 0.0f, m2 = 0.7939f, m3 = -0.6065f, m4 = 0.3539f, m5 = 0.6373f, m6 = 0.5995f;
            T alpha = -1.0f * M<T>::log10(M<T>::exp((T)1.0f)) / m4;
            T beta_ = M<T>::exp(m3 / m4);
            T k = (T)(2 * REF_PI / (c[i] * Trep));
            T Ur = 3.0f / 8.0f * M<T>::sqrt((T)2.0f) * H[i] * k / M<T>::pow(k * hh[i], 3.0f);
            Ur = M<T>::fmax(Ur, 0.00001f);
            T Bm = m1 + (m2 - m1) / (1.0f + beta_ * M<T>::pow(Ur, alpha));
            T B1 = (T)((-90.0f + 90.0f * M<T>::tanh(m5 / M<T>::pow(Ur, m6))) * REF_PI / 180.0f);
            T Sk = Bm * M<T>::cos(B1);
            T As = Bm * M<T>::sin(B1);
            ua[i] = (facsk * Sk - facas * As) * urms[i];
        }
        /* Erosus (:512-531) */
        T morfac = (T)P.morfac, por = (T)P.por;
        for (int i = 0; i < C; i++) {
            T pbbed = 1.0f;
            T exp_ero = morfac * dtf / (1.0f - por) * hh[i] * (ceqsg[i] * pbbed / Tsg[i] + ceqbg[i] * pbbed / dtf);
            facero[i] = M<T>::fmin(1.0f, stdep[i] * pbbed / M<T>::fmax(0.000001f, exp_ero));
        }
        /* Susp (:534-719) */
        T sus = (T)P.sus;
        for (int iy = 0; iy < ny; iy++)
            for (int ix = 0; ix < nx; ix++) {
                int i = I(ix, iy);
                int xp = pp(ix, nx), yp = pp(iy, ny);
                T facsl = 1.6f;
                T hhi = hh[i], zbi = zb[i], zbr = zb[I(xp, iy)], zbt = zb[I(ix, yp)];
                T cci = Cc[i], ccr = Cc[I(xp, iy)], cct = Cc[I(ix, yp)];
                T uui = uu[i], vvi = vv[i];
                T tm = thm[i];
                T uau = (T)(0.5 * M<T>::cos(tm) * (ua[i] + ua[I(xp, iy)]));
                T uav = (T)(0.5 * M<T>::sin(tm) * (ua[I(xp, iy)] + ua[i]));
                T uv = uvg[i], vu = vug[i];
                T urep = ueu[i] + uau;
                T vmagu = M<T>::sqrt(M<T>::pow((uui + uau), 2.0f) + M<T>::pow((vu + uav), 2.0f));
                uau = (T)(0.5 * M<T>::cos(tm) * (ua[i] + ua[I(ix, yp)]));
                uav = (T)(0.5 * M<T>::sin(tm) * (ua[I(ix, yp)] + ua[i]));
                T vrep = vev[i] + uav;
                T vmagv = M<T>::sqrt(M<T>::pow(uv + uau, 2.0f) + M<T>::pow(vvi + uav, 2.0f));
                T dzbdx = -1.0f * (zbr - zbi) / dx;
                T dzbdy = -1.0f * (zbt - zbi) / dx;
                T hui = hu[i], hvi = hv[i];
                T wu_ = hui > eps ? 1.0f : 0.0f;
                T wv_ = hvi > eps ? 1.0f : 0.0f;
                T cu, cv;
                if (urep > 0.0f) cu = cci;
                else if (urep < 0.0f) cu = ccr;
                else cu = 0.50f * (cci + ccr);
                T dcsdx = (ccr - cci) / dx;
                if (vrep > 0.0f) cv = cci;
                else if (vrep < 0.0f) cv = cct;
                else cv = 0.50f * (cci + cct);
                T dcsdy = (cct - cci) / dx;
                T Dc = nuh + nuhfac * hhi * M<T>::pow(DR[i] / rho, 1.0f / 3.0f);
                Sus[i] = sus * (cu * urep * hui - Dc * hui * dcsdx - facsl * cu * vmagu * hui * dzbdx) * wu_;
                Svs[i] = sus * (cv * vrep * hvi - Dc * hvi * dcsdy - facsl * cv * vmagv * hvi * dzbdy) * wv_;
            }
        /* Conc (:721-780) */
        for (int iy = 0; iy < ny; iy++)
            for (int ix = 0; ix < nx; ix++) {
                int i = I(ix, iy);
                T hhi = hh[i];
                T wetz = hhi > eps ? 1.0f : 0.0f;
                T Pbed = 1.0f;
                ero[i] = facero[i] * hhi * ceqsg[i] * Pbed / Tsg[i];
                T dsusdx = (Sus[i] - Sus[I(mm(ix), iy)]) / dx;
                T dsvsdy = (Svs[i] - Svs[I(ix, mm(iy))]) / dx;
                T cs = (dtf * Tsg[i]) / (dtf + Tsg[i]) * (hhi * Cc[i] / dtf - (dsusdx + dsvsdy - ero[i])) * wetz;
                cs = M<T>::fmax(cs, 0.0f);
                cs = M<T>::fmin(cs, 0.1f * hhi);
                depo[i] = cs / Tsg[i];
                Cc[i] = cs / hh[i];
            }
        /* CClatbnd (:782-821) */
        {
            std::vector<T> o(Cc, Cc + C);
            for (int iy = 0; iy < ny; iy++)
                for (int ix = 0; ix < nx; ix++) {
                    int i = I(ix, iy);
                    if (iy == 0) Cc[i] = o[I(ix, pp(iy, ny))];
                    if (iy == ny - 1) Cc[i] = o[I(ix, mm(iy))];
                    if (ix == 0) Cc[i] = 0.0f;
                }
        }
        if (P.morfac > 0.0f) {
            /* bedupdate (:881-968) */
            for (int i = 0; i < C; i++) {
                T dzg = morfac * dtf / (1.0f - por) * (ero[i] - depo[i]);
                zb[i] = zb[i] + dzg;
                hh[i] = hh[i] + dzg;
                dzb[i] = -1 * dzg;
                stdep[i] = stdep[i] - dzg;
            }
            zblatbnd(zb);
            zblatbnd(stdep);
            /* avalanching (:1020-1137), gathered (deviation 4) */
            T drydzmax = (T)P.drydzmax, wetdzmax = (T)P.wetdzmax, maxchg = (T)P.maxslpchg;
            std::vector<T> ax(C), ay(C);
            for (int iy = 0; iy < ny; iy++)
                for (int ix = 0; ix < nx; ix++) {
                    int i = I(ix, iy);
                    int xp = pp(ix, nx), yp = pp(iy, ny);
                    T Zbi = zb[i], Zbt = zb[I(ix, yp)], Zbr = zb[I(xp, iy)];
                    T sti = stdep[i], stt = stdep[I(ix, yp)], str = stdep[I(xp, iy)];
                    T dzmax = hh[i] > eps ? wetdzmax : drydzmax;
                    T dzbx = 0.0f, dzby = 0.0f;
                    T dzbdx = (Zbr - Zbi) / dx;
                    if (M<T>::fabs(dzbdx) > dzmax) {
                        T s = dzbdx / M<T>::fabs(dzbdx);
                        dzbx = s * (M<T>::fabs(dzbdx) - dzmax) * dx;
                        if (s > 0) {
                            dzbx = M<T>::fmin(dzbx, maxchg * dtf / dx);
                            dzbx = M<T>::fmin(dzbx, sti);
                        } else {
                            dzbx = M<T>::fmax(dzbx, -1.0f * maxchg * dtf / dx);
                            dzbx = M<T>::fmax(dzbx, -1.0f * str);
                        }
                    }
                    T dzbdy = (Zbt - Zbi) / dx;
                    if (M<T>::fabs(dzbdy) > dzmax) {
                        T s = dzbdy / M<T>::fabs(dzbdy);
                        dzby = s * (M<T>::fabs(dzbdy) - dzmax) * dx;
                        if (s > 0) {
                            dzby = M<T>::fmin(dzby, maxchg * dtf / dx);
                            dzby = M<T>::fmin(dzby, sti);
                        } else {
                            dzby = M<T>::fmax(dzby, -1 * maxchg * dtf / dx);
                            dzby = M<T>::fmax(dzby, -1 * stt);
                        }
                    }
                    ax[i] = dzbx; ay[i] = dzby;
                }
            for (int iy = 0; iy < ny; iy++)
                for (int ix = 0; ix < nx; ix++) {
                    int i = I(ix, iy);
                    T a = 0.0f;
                    if (iy > 0) a = a - ay[I(ix, iy - 1)];
                    if (ix > 0) a = a - ax[I(ix - 1, iy)];
                    a = a + ax[i];
                    a = a + ay[i];
                    ddzb[i] = a;
                }
            /* updatezb (:1139-1160) */
            for (int i = 0; i < C; i++) {
                zb[i] = zb[i] + ddzb[i];
                dzb[i] = dzb[i] - ddzb[i];
                zs[i] = zs[i] - ddzb[i];
                stdep[i] = stdep[i] - ddzb[i];
                hh[i] = hh[i] - ddzb[i];
            }
            zblatbnd(zb);
            zblatbnd(stdep);
            updatezom();
        }
        return XBG_OK;
    }

    /* ====================================================== running means */
    int means() override {   /* Wave_gpu.cu:731-757 */
        if (status != XBG_OK) return status;
        const T* H = f(XBG_F_H); const T* uu = f(XBG_F_UU); const T* vv = f(XBG_F_VV);
        const T* hh = f(XBG_F_HH); const T* zs = f(XBG_F_ZS); const T* Cc = f(XBG_F_CC);
        T* Hm = f(XBG_F_HMEAN); T* um = f(XBG_F_UUMEAN); T* vm = f(XBG_F_VVMEAN);
        T* hm = f(XBG_F_HHMEAN); T* zm = f(XBG_F_ZSMEAN); T* zx = f(XBG_F_ZSMAX);
        T* cm = f(XBG_F_CMEAN);
        for (int i = 0; i < C; i++) {
            Hm[i] = Hm[i] + H[i]; um[i] = um[i] + uu[i]; vm[i] = vm[i] + vv[i];
            hm[i] = hm[i] + hh[i]; zm[i] = zm[i] + zs[i];
            zx[i] = M<T>::fmax(zx[i], zs[i]);
            cm[i] = cm[i] + Cc[i];
        }
        return XBG_OK;
    }
    int output_done() override {   /* Wave_gpu.cu:786-824 */
        nextoutputtime = nextoutputtime + P.outputtimestep;
        T nd = (T)nstep;
        int ids[] = {XBG_F_HMEAN, XBG_F_UUMEAN, XBG_F_VVMEAN, XBG_F_HHMEAN, XBG_F_ZSMEAN, XBG_F_CMEAN};
        for (int id : ids)
            for (int i = 0; i < C; i++) F[id][i] = F[id][i] / nd;
        flags &= ~XBG_FLAG_OUTPUT_DUE;
        return XBG_OK;
    }
    int reset_means() override {   /* Wave_gpu.cu:894-928 */
        int ids[] = {XBG_F_HMEAN, XBG_F_UUMEAN, XBG_F_VVMEAN, XBG_F_HHMEAN, XBG_F_ZSMEAN, XBG_F_ZSMAX, XBG_F_CMEAN};
        for (int id : ids) std::fill(F[id].begin(), F[id].end(), (T)0);
        nstep = 0;
        return XBG_OK;
    }
    void mass(double* w, double* s, double* b) override {
        double a = P.dx * P.dx, sw = 0, ss = 0, sb = 0;
        const T* zs = f(XBG_F_ZS); const T* hh = f(XBG_F_HH);
        const T* Cc = f(XBG_F_CC); const T* zb = f(XBG_F_ZB);
        for (int i = 0; i < C; i++) {
            sw += (double)zs[i]; ss += (double)Cc[i] * (double)hh[i]; sb += (double)zb[i];
        }
        *w = sw * a; *s = ss * a; *b = sb * a;
    }
};

}  // namespace

/* ============================================================== C API */
extern "C" {

int xbgo_create(const xbg_params* p, int precision, xbgo** out) {
    if (!p || !out || p->nx < 4 || p->ny < 4 || p->ntheta < 1) return XBG_ERR_ARG;
    if (precision == XBG_FP32) *out = new Oracle<float>(p, precision);
    else if (precision == XBG_FP64) *out = new Oracle<double>(p, precision);
    else return XBG_ERR_ARG;
    return XBG_OK;
}
int xbgo_destroy(xbgo* o) { delete o; return XBG_OK; }
int xbgo_init_state(xbgo* o, const void* zb, double zs0, double zs1) { return o->init_state(zb, zs0, zs1); }
int xbgo_field_count(const xbgo* o, int f, size_t* n) { return o->field_count(f, n); }
int xbgo_set_field(xbgo* o, int f, const void* p, size_t n) { return o->set_field(f, p, n); }
int xbgo_get_field(xbgo* o, int f, void* p, size_t n) { return o->get_field(f, p, n); }

int xbgo_set_wave_boundary(xbgo* o, int slot, const double* St, const double* q, int nrec,
                           const double* times, double t0, double tend, double Trep) {
    if (slot < 0 || slot > 1 || nrec < 2 || !St || !q) return XBG_ERR_ARG;
    Chunk c;
    c.valid = true; c.nrec = nrec; c.t0 = t0; c.tend = tend; c.Trep = Trep;
    size_t ns = (size_t)nrec * o->P.ntheta * o->P.ny, nq = (size_t)nrec * 4 * o->P.ny;
    c.St.assign(St, St + ns);
    c.q.assign(q, q + nq);
    if (times) c.times.assign(times, times + nrec);
    else { c.times.resize(nrec); for (int m = 0; m < nrec; m++) c.times[m] = t0 + m * o->P.dtbc; }
    o->chunk[slot] = c;
    if (slot == 1) o->flags &= ~XBG_FLAG_NEED_BOUNDARY;
    return XBG_OK;
}
int xbgo_set_sealevel(xbgo* o, const double* t, const double* a, const double* b, int n) {
    if (n < 2) return XBG_ERR_ARG;
    o->sl.t.assign(t, t + n); o->sl.a.assign(a, a + n); o->sl.b.assign(b, b + n);
    o->SLstep = 1;
    return XBG_OK;
}
int xbgo_set_wind(xbgo* o, const double* t, const double* a, const double* b, int n) {
    if (n < 2) return XBG_ERR_ARG;
    o->wnd.t.assign(t, t + n); o->wnd.a.assign(a, a + n); o->wnd.b.assign(b, b + n);
    o->WNDstep = 1;
    return XBG_OK;
}
int xbgo_compute_dt(xbgo* o) { return o->compute_dt(); }
int xbgo_wave_boundary(xbgo* o) { return o->wave_boundary(); }
int xbgo_flow_boundary(xbgo* o) { return o->flow_boundary(); }
int xbgo_wave_step(xbgo* o) { return o->wave_step(); }
int xbgo_flow_step(xbgo* o) { return o->flow_step(); }
int xbgo_sediment_step(xbgo* o) { return o->sediment_step(); }
int xbgo_accumulate_means(xbgo* o) { return o->means(); }

int xbgo_step(xbgo* o) {   /* one mainloopGPU iteration, Wave_gpu.cu:610-782 */
    int s;
    if ((s = o->compute_dt())) return s;
    if (o->P.swave == 1 && (s = o->wave_boundary())) return s;
    if (o->P.flow == 1 && (s = o->flow_boundary())) return s;
    if (o->P.swave == 1 && (s = o->wave_step())) return s;
    if (o->P.flow == 1 && (s = o->flow_step())) return s;
    if ((s = o->sediment_step())) return s;
    if (o->P.means && (s = o->means())) return s;
    if (o->nextoutputtime - o->totaltime <= o->dt * 0.001 && o->P.outputtimestep > 0)
        o->flags |= XBG_FLAG_OUTPUT_DUE;
    if (o->totaltime >= o->P.endtime) o->flags |= XBG_FLAG_ENDED;
    return XBG_OK;
}
int xbgo_advance(xbgo* o, int nsteps) {
    for (int k = 0; k < nsteps; k++) {
        if (o->status != XBG_OK) return o->status;
        if (o->flags & (XBG_FLAG_OUTPUT_DUE | XBG_FLAG_ENDED)) break;
        int s = xbgo_step(o);
        if (s) return s;
    }
    return XBG_OK;
}
int xbgo_get_time(xbgo* o, double* t, double* dt, int64_t* n, int* flags) {
    if (t) *t = o->totaltime;
    if (dt) *dt = o->dt;
    if (n) *n = o->nstep_total;
    if (flags) *flags = o->flags;
    return o->status;
}
int xbgo_set_time(xbgo* o, double t, double dt, double wdt) {
    o->totaltime = t; o->dt = dt; o->wdt = wdt;
    return XBG_OK;
}
int xbgo_output_done(xbgo* o) { return o->output_done(); }
int xbgo_reset_means(xbgo* o) { return o->reset_means(); }
int xbgo_mass(xbgo* o, double* w, double* s, double* b) { o->mass(w, s, b); return XBG_OK; }

}  // extern "C"
