// wavegen.cu -- offshore wave-boundary records from a JONSWAP spectrum:
// wave-group energy per directional bin (St) and bound long-wave fluxes (q),
// the algorithm of makjonswap + GenWGnLBW (makjonswap.cpp:73-1419).
//
// Host set-up (serial, O(K * spectrum size)): the spectrum, the component
// frequency range and count K, random phases and directions (drawn with
// std::default_random_engine / uniform_real_distribution in the reference's
// order), wave numbers, Trep, the internal time axis and tapers, component
// variances and directional bins.
//
// Device (double precision):
//   k_wg_coef   G_c(j) = a_c e^{i phi_c} e^{-i k_c sin(theta_c) j dx}, the
//               Fourier coefficient of component c at offshore point j
//   k_wg_zeta   the surface elevation of each directional bin at every
//               internal time step: the inverse DFT of the bin's Hermitian
//               coefficient array, evaluated as the sum over its components
//               (2 Re(G e^{2 pi i F n / N})), times the wave taper; the sum
//               over bins (eta) and per-block sums of squares
//   k_wg_std    standard deviations of eta and of each bin's elevation
//   k_wg_fft*   the Hilbert envelope of eta: zero-padded radix-2 FFT,
//               one-sided weights, inverse FFT (global memory, all offshore
//               points at once)
//   k_wg_st     St at the record times: (|analytic eta| std_bin / std_eta)^2
//               rho g / (2 dtheta), linearly interpolated in time
//   k_wg_pairs  difference-interaction coefficients of every component pair
//               (Herbers 1994, Van Dongeren et al. 2003), as the reference
//               evaluates them
//   k_wg_bound  per offshore point and difference frequency, the sum over
//               pairs of the bound-wave flux coefficients unrolled along the
//               boundary
//   k_wg_q      q at the record times: inverse DFT of those coefficients at
//               the two bracketing internal steps, tapered, interpolated.
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdio>
#include <random>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/xbg_bnd.h"

namespace {

const double PI_R = 3.14159265;   // the reference's pi macro

// ---------------------------------------------------------------- host helpers
// Linear search interpolation (tools.cpp:28-62): the interval ends at the
// first abscissa >= xx; beyond the last one the first interval is used.
double interp_search(int n, const double* x, const double* y, double xx) {
    int lo = 0;
    for (int i = 0; i < n; i++)
        if (xx - x[i] <= 0.0) { lo = i - 1 > 0 ? i - 1 : 0; break; }
    const int hi = lo + 1 < n - 1 ? lo + 1 : n - 1;
    return y[lo] + (xx - x[lo]) / (x[hi] - x[lo]) * (y[hi] - y[lo]);
}
// Interpolation on a uniform axis (tools.cpp:64-91).
double interp_uniform(int n, const double* x, const double* y, double xx) {
    const double dx = x[1] - x[0];
    const double d = xx - x[0] > 0.0 ? xx - x[0] : 0.0;
    const int lo = (int)std::floor(d / dx);
    const int hi = lo + 1 < n - 1 ? lo + 1 : n - 1;
    return y[lo] + (xx - x[lo]) / (x[hi] - x[lo]) * (y[hi] - y[lo]);
}
int search_lo(int n, const double* x, double xx) {
    for (int i = 0; i < n; i++)
        if (xx - x[i] <= 0.0) return i - 1 > 0 ? i - 1 : 0;
    return 0;
}
// Bilinear interpolation of z[ix + iy*nx] (tools.cpp:93-161).
double interp_bilinear(int nx, int ny, const double* x, const double* y, const double* z, double xx, double yy) {
    const int ix = search_lo(nx, x, xx), ixp = ix + 1 < nx - 1 ? ix + 1 : nx - 1;
    const int iy = search_lo(ny, y, yy), iyp = iy + 1 < ny - 1 ? iy + 1 : ny - 1;
    const double x1 = x[ix], x2 = x[ixp], y1 = y[iy], y2 = y[iyp];
    const double q11 = z[ix + iy * nx], q12 = z[ix + iyp * nx], q21 = z[ixp + iy * nx], q22 = z[ixp + iyp * nx];
    return 1.0 / ((x2 - x1) * (y2 - y1)) *
           (q11 * (x2 - xx) * (y2 - yy) + q21 * (xx - x1) * (y2 - yy) + q12 * (x2 - xx) * (yy - y1) +
            q22 * (xx - x1) * (yy - y1));
}
double dmax(double a, double b) { return (a < b) ? b : a; }
double dmin(double a, double b) { return !(b < a) ? a : b; }

// The JONSWAP frequency-direction spectrum S[f + d*nf] [m2/Hz/rad] on 90
// directions over the full circle (makjonswap.cpp:73-233).
struct Spectrum {
    int nf = 0, nd = 0;
    std::vector<double> f, d, S;
};
Spectrum jonswap(double Hs, double Tp_in, double mainang, double s_in, double gam) {
    Spectrum sp;
    const double Tp = dmax(Tp_in, 1.5);
    const double fp = 1 / Tp;
    const double scoeff = dmax(std::round(dmin(s_in, 1000.0)), 10.0);
    const double fnyq = 3.0f * fp, dfj = fp / 20.0f;
    sp.nf = (int)std::ceil((fnyq - dfj) / dfj);
    sp.f.resize(sp.nf);
    std::vector<double> y(sp.nf);
    double ysum = 0.0, ymax = 0.0;
    for (int i = 0; i < sp.nf; i++) {
        sp.f[i] = (i + 1) * dfj;
        double xa = std::abs(sp.f[i] / fp);
        if (xa == 0) xa = 1e-7f;
        const double sig = xa < 1 ? 0.07f : 0.09f;
        const double g1 = std::pow(xa, -5);
        const double g2 = std::exp(-1.25 * std::pow(xa, -4.0f));
        const double g3 = std::pow(gam, std::exp(-(std::pow(xa - 1.0f, 2) / (2 * std::pow(sig, 2)))));
        y[i] = g1 * g2 * g3;
        ysum = ysum + y[i];
        if (y[i] >= ymax) ymax = y[i];
    }
    ysum = ysum / ymax;
    for (int i = 0; i < sp.nf; i++) {
        y[i] = y[i] / ymax;
        y[i] = y[i] * std::pow(Hs / (4 * std::sqrt(ysum * dfj)), 2);
    }
    sp.nd = 90;
    const double dth = 2 * PI_R / sp.nd;
    sp.d.resize(sp.nd);
    std::vector<double> Dd(sp.nd);
    double ddsum = 0.0;
    for (int i = 0; i < sp.nd; i++) {
        sp.d[i] = i * dth - PI_R;
        Dd[i] = std::pow(std::cos((sp.d[i] - mainang) / 2.0f), 2.0 * scoeff);
        ddsum = ddsum + Dd[i];
    }
    const double dang = sp.d[1] - sp.d[0];
    for (int i = 0; i < sp.nd; i++) Dd[i] = Dd[i] / (ddsum * dang);
    sp.S.resize((size_t)sp.nf * sp.nd);
    for (int i = 0; i < sp.nd; i++)
        for (int k = 0; k < sp.nf; k++) sp.S[k + (size_t)i * sp.nf] = y[k] * Dd[i];
    return sp;
}

// ---------------------------------------------------------------- device
struct Pair {   // bound-wave coefficients of pair (i, m): flux factors and unrolling
    double fxr, fxi, fyr, fyi, kky;
};

// G_c(j) = (ar + i ai) (cos b - i sin b), b = k_c (sin(theta_c) (j dx))
__global__ void k_wg_coef(const double* ar, const double* ai, const double* kc, const double* sc, int K, int ny,
                          double dx, double2* G) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y;
    if (c >= K) return;
    double sb, cb;
    sincos(kc[c] * (sc[c] * (j * dx)), &sb, &cb);
    G[(size_t)j * K + c] = make_double2(ar[c] * cb + ai[c] * sb, ai[c] * cb - ar[c] * sb);
}

// twiddle index (F n) mod N with 32-bit arithmetic (N <= 65535)
__device__ __forceinline__ unsigned tw(unsigned F, unsigned n, unsigned N) { return (F * n) % N; }

// one thread per internal time step n of offshore point j = blockIdx.y; the
// block's sums of squares of each bin b (and of eta, b = nbin) go to
// part[(j * (nbin + 1) + b) * nblk + blockIdx.x]
constexpr int WG_T = 256;
constexpr int WG_MAXBIN = 64;
__global__ void __launch_bounds__(WG_T) k_wg_zeta(const double2* G, const int* F, const int* bstart,
                                                  const int* bcount, int K, int nbin, int N, const double2* W,
                                                  const double* taperw, double* eta, double* part) {
    __shared__ double red[WG_T / 32];
    const int j = blockIdx.y, n = blockIdx.x * WG_T + threadIdx.x;
    const bool live = n < N;
    const double2* Gj = G + (size_t)j * K;
    const double tp = live ? taperw[n] : 0.0;
    double e = 0.0;
    for (int b = 0; b < nbin; b++) {
        double z = 0.0;
        if (live) {
            const int c0 = bstart[b], c1 = c0 + bcount[b];
            for (int c = c0; c < c1; c++) {
                const unsigned f = (unsigned)F[c];
                const double2 w = W[tw(f, (unsigned)n, (unsigned)N)];
                const double2 g = Gj[c];
                const double re = g.x * w.x - g.y * w.y;
                z += (f == 0 || 2 * f == (unsigned)N) ? re : 2.0 * re;
            }
            z = z * tp;
        }
        e = e + z;
        // block sum of z^2 in a fixed order
        double v = z * z;
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
        __syncthreads();
        if (threadIdx.x == 0) {
            double s = 0.0;
            for (int w = 0; w < WG_T / 32; w++) s += red[w];
            part[((size_t)j * (nbin + 1) + b) * gridDim.x + blockIdx.x] = s;
        }
        __syncthreads();
    }
    if (live) eta[(size_t)j * N + n] = e;
    double v = e * e;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < WG_T / 32; w++) s += red[w];
        part[((size_t)j * (nbin + 1) + nbin) * gridDim.x + blockIdx.x] = s;
    }
}

// std = sqrt(sum / (N - 1)) of each bin (b < nbin) and of eta (b = nbin)
__global__ void k_wg_std(const double* part, int nblk, int nbin, int ny, int N, double* sd) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ny * (nbin + 1)) return;
    double s = 0.0;
    for (int k = 0; k < nblk; k++) s += part[(size_t)t * nblk + k];
    sd[t] = sqrt(s / (N - 1));
}

// ---- radix-2 FFT of every row of X [ny][n2] (in place, global memory)
__global__ void k_wg_fft_load(const double* eta, int N, int n2, int logn, int ny, double2* X) {
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (size_t)ny * n2) return;
    const int j = (int)(t / n2), k = (int)(t % n2);
    const unsigned r = __brev((unsigned)k) >> (32 - logn);
    X[(size_t)j * n2 + r] = make_double2(k < N ? eta[(size_t)j * N + k] : 0.0, 0.0);
}
// one butterfly stage; sign -1 forward, +1 backward; W2[m] = e^{2 pi i m / n2}
__global__ void k_wg_fft_stage(double2* X, int n2, int half, int ny, const double2* W2, int sign) {
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const size_t nb = (size_t)n2 / 2;
    if (t >= (size_t)ny * nb) return;
    const int j = (int)(t / nb), b = (int)(t % nb);
    const int grp = b / half, pos = b % half;
    const int i0 = grp * 2 * half + pos, i1 = i0 + half;
    const double2 w0 = W2[pos * (n2 / (2 * half))];
    const double2 w = make_double2(w0.x, sign * w0.y);
    double2* r = X + (size_t)j * n2;
    const double2 a = r[i0], c = r[i1];
    const double2 tt = make_double2(w.x * c.x - w.y * c.y, w.x * c.y + w.y * c.x);
    r[i0] = make_double2(a.x + tt.x, a.y + tt.y);
    r[i1] = make_double2(a.x - tt.x, a.y - tt.y);
}
// one-sided weights h (1, 2 ... 2, 1, 0 ... 0) and the bit-reversed reload
// for the inverse transform
__global__ void k_wg_fft_hilbert(const double2* X, int n2, int logn, int ny, double2* Y) {
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (size_t)ny * n2) return;
    const int j = (int)(t / n2), k = (int)(t % n2);
    const double h = (k == 0 || k == n2 / 2) ? 1.0 : (k < n2 / 2 ? 2.0 : 0.0);
    const double2 v = X[t];
    const unsigned r = __brev((unsigned)k) >> (32 - logn);
    Y[(size_t)j * n2 + r] = make_double2(v.x * h, v.y * h);
}
// |analytic signal| of the first N samples
__global__ void k_wg_fft_amp(const double2* Y, int N, int n2, int ny, double* amp) {
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (size_t)ny * N) return;
    const int j = (int)(t / N), k = (int)(t % N);
    const double2 v = Y[(size_t)j * n2 + k];
    const double re = v.x / n2, im = v.y / n2;
    amp[t] = hypot(re, im);
}

// St[m][b][j]: the energy series of bin b at offshore point j interpolated to
// the record time m dtbc (interp_uniform on the internal axis n dtin)
__global__ void k_wg_st(const double* amp, const double* sd, int nbin, int ny, int N, int nrec, double dtbc,
                        double dtin, double rho, double g, double dtheta, double* St, int* bad) {
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (size_t)nrec * nbin * ny) return;
    const int j = (int)(t % ny), b = (int)((t / ny) % nbin), m = (int)(t / ((size_t)ny * nbin));
    const double se = sd[(size_t)j * (nbin + 1) + nbin], sb = sd[(size_t)j * (nbin + 1) + b];
    const double xx = m * dtbc;
    const double x0 = 0 * dtin, x1 = 1 * dtin;
    const double d = xx - x0 > 0.0 ? xx - x0 : 0.0;
    const int lo = (int)floor(d / (x1 - x0));
    const int hi = lo + 1 < N - 1 ? lo + 1 : N - 1;
    auto E = [&](int n) {
        const double z = se > 0.0 ? amp[(size_t)j * N + n] * sb / se : 0.0;
        return z * z * 0.5 * rho * g / (dtheta);
    };
    const double xl = lo * dtin, xh = hi * dtin;
    const double el = E(lo), eh = E(hi);
    const double v = el + (xx - xl) / (xh - xl) * (eh - el);
    if (v != v) atomicExch(bad, 1);
    St[t] = v;
}

struct PairIn {   // per component: wave number, angular frequency, direction, frequency, variance
    const double *k, *w, *th, *f, *vq, *arg;
};
// coefficients of pair (i = 1..K-1, m = 0..K-i-1) at [(i-1) * K + m]
__global__ void k_wg_pairs(PairIn P, int K, double dfgen, double g, double h, double nmax, double fcutoff,
                           Pair* out) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y + 1;
    if (m >= K - i) return;
    const double deltaf = (i + 1) * dfgen;
    const int mi = i + m;
    const double km = P.k[m], kmi = P.k[mi];
    const double deltatheta = fabs(P.th[mi] - P.th[m]) + PI_R;
    const double KKy = kmi * sin(P.th[mi]) - km * sin(P.th[m]);
    const double KKx = kmi * cos(P.th[mi]) - km * cos(P.th[m]);
    const double cdt = cos(deltatheta);
    const double k3 = sqrt(km * km + kmi * kmi + 2 * km * kmi * cdt);
    double cg3 = 2 * PI_R * deltaf / k3;
    const double cap = nmax * sqrt(g / k3 * tanh(k3 * h));
    cg3 = !(cap < cg3) ? cg3 : cap;
    const double wm = P.w[m], wmi = P.w[mi];
    const double t1 = (-1.0 * wm) * wmi;
    const double t2 = (-1.0 * wm) + wmi;
    const double t2n = cg3 * k3;
    const double chk1 = cosh(km * h), chk2 = cosh(kmi * h);
    double D = -1.0 * g * km * kmi * cdt * 0.5 / t1 +
               g * t2 * (chk1 * chk2) / ((g * k3 * tanh(k3 * h) - t2n * t2n) * t1 * cosh(k3 * h)) *
                   (t2 * (t1 * t1 / (g * g) - km * kmi * cdt) -
                    0.5 * ((-1.0 * wm) * kmi * kmi / (chk2 * chk2) + wmi * km * km / (chk1 * chk1)));
    D = D * cosh(k3 * h) / (cosh(km * h) * cosh(kmi * h));
    if (P.f[m] <= deltaf) D = 0.0;
    if (deltaf <= fcutoff) D = 0.0;
    // phase from the coefficients of components mi-1 and m-1 (arg[c + 1];
    // arg[0] stands for the empty slot below the first component)
    const double dphi3 = PI_R + P.arg[mi] - P.arg[m];
    const double theta3 = atan2(KKy, KKx);
    const double Eforc = 2 * D * D * P.vq[m] * P.vq[mi] * dfgen;
    const double Abnd = sqrt(2.0 * Eforc * dfgen);
    double sp, cp;
    sincos(dphi3, &sp, &cp);
    // Abnd 0.5 e^{-i dphi3} cg3 cos(theta3) and ... sin(theta3), left to right
    const double ar = Abnd * 0.50 * cp, ai = Abnd * 0.50 * -sp;
    const double ct = cos(theta3), st = sin(theta3);
    Pair p;
    p.fxr = ar * cg3 * ct; p.fxi = ai * cg3 * ct;
    p.fyr = ar * cg3 * st; p.fyi = ai * cg3 * st;
    p.kky = KKy;
    out[(size_t)(i - 1) * K + m] = p;
}

// Gq[j][i] = sum over m of the pair (i, m) flux factors unrolled to offshore
// point j: (qx, qy) coefficient of difference frequency index i
__global__ void k_wg_bound(const Pair* P, int K, int ny, double dx, double4* Gq) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y + 1;
    if (j >= ny) return;
    double xr = 0, xi = 0, yr = 0, yi = 0;
    const Pair* row = P + (size_t)(i - 1) * K;
    for (int m = 0; m < K - i; m++) {
        const Pair p = row[m];
        double s, c;
        sincos(-(p.kky * (j * dx) + 0.0), &s, &c);
        xr += p.fxr * c - p.fxi * s; xi += p.fxr * s + p.fxi * c;
        yr += p.fyr * c - p.fyi * s; yi += p.fyr * s + p.fyi * c;
    }
    Gq[(size_t)j * K + i] = make_double4(xr, xi, yr, yi);
}

// q[m][c][j]: qx (c = 0) and qy (c = 1) at the record times, c = 2, 3 zero
__global__ void k_wg_q(const double4* Gq, int K, int ny, int N, const double2* W, const double* taperf, int nrec,
                       double dtbc, double dtin, double* q) {
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (size_t)nrec * ny) return;
    const int j = (int)(t % ny), m = (int)(t / ny);
    const double xx = m * dtbc;
    const double d = xx > 0.0 ? xx : 0.0;
    const int lo = (int)floor(d / (1 * dtin - 0 * dtin));
    const int hi = lo + 1 < N - 1 ? lo + 1 : N - 1;
    const double4* g = Gq + (size_t)j * K;
    auto synth = [&](int n, double& qx, double& qy) {
        double ax = 0.0, ay = 0.0;
        for (int i = 1; i < K; i++) {
            const double4 v = g[i];
            const double2 w = W[tw((unsigned)i, (unsigned)n, (unsigned)N)];
            ax += 2.0 * (v.x * w.x - v.y * w.y);
            ay += 2.0 * (v.z * w.x - v.w * w.y);
        }
        qx = ax * taperf[n];
        qy = ay * taperf[n];
    };
    double qxl, qyl, qxh, qyh;
    synth(lo, qxl, qyl);
    synth(hi, qxh, qyh);
    const double xl = lo * dtin, xh = hi * dtin;
    double* o = q + (size_t)m * 4 * ny;
    o[j] = qxl + (xx - xl) / (xh - xl) * (qxh - qxl);
    o[j + ny] = qyl + (xx - xl) / (xh - xl) * (qyh - qyl);
    o[j + 2 * ny] = 0.0;
    o[j + 3 * ny] = 0.0;
}

// twiddles e^{2 pi i m / n}, m < n, from long-double cos/sin of the reduced angle
std::vector<double2> twiddles(int n) {
    std::vector<double2> w(n);
    const long double tp = 6.283185307179586476925286766559L;
    for (int m = 0; m < n; m++) {
        const long double a = tp * (long double)m / (long double)n;
        w[m] = make_double2((double)cosl(a), (double)sinl(a));
    }
    return w;
}

struct DevBufs {
    std::vector<void*> p;
    ~DevBufs() { for (void* q : p) cudaFree(q); }
    template <class T> T* get(size_t n) {
        void* q = nullptr;
        if (cudaMalloc(&q, (n ? n : 1) * sizeof(T)) != cudaSuccess) return nullptr;
        p.push_back(q);
        return (T*)q;
    }
    template <class T> T* put(const std::vector<T>& v) {
        T* d = get<T>(v.size());
        if (d && !v.empty() && cudaMemcpy(d, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess)
            return nullptr;
        return d;
    }
};

}  // namespace

extern "C" void xbg_wavegen_default(xbg_wavegen* w) {
    if (!w) return;
    w->Hs = 1.0; w->Tp = 10.0; w->Dp = 0.0; w->s = 10.0; w->gamma = 3.3;
    w->sprdthr = 0.08; w->offdepth = 10.0; w->nmax = 0.8; w->fcutoff = 0.0; w->nspr = 0; w->seed = 0;
}

extern "C" int xbg_gen_wave_groups(const xbg_params* p, const xbg_wavegen* w, double* St, double* q, int nrec,
                                   double* Trep) {
    if (!p || !w || !St || !q || !Trep || p->ny < 1 || p->ntheta < 1 || p->ntheta > WG_MAXBIN || p->dtbc <= 0 ||
        p->rtlength <= 0 || w->offdepth <= 0)
        return XBG_ERR_ARG;
    const int ny = p->ny, nbin = p->ntheta;
    const int tslenbc = (int)std::ceil(p->rtlength / p->dtbc) + 1;
    if (nrec != tslenbc) return XBG_ERR_ARG;
    // ---- spectrum, frequency and direction integrals (makjonswap.cpp:270-303)
    const Spectrum sp = jonswap(w->Hs, w->Tp, w->Dp, w->s, w->gamma);
    const int nf = sp.nf, nd = sp.nd;
    const double dtheta = sp.d[1] - sp.d[0], dfreq = sp.f[1] - sp.f[0];
    std::vector<double> Sf(nf);
    double Hm0 = 0.0;
    for (int n = 0; n < nf; n++) {
        Sf[n] = 0.0;
        for (int d = 0; d < nd; d++) Sf[n] = Sf[n] + sp.S[n + (size_t)d * nf];
        Sf[n] = Sf[n] * dtheta;
        Hm0 = Hm0 + Sf[n];
    }
    Hm0 = 4.0 * std::sqrt(Hm0 * dfreq);
    // ---- component frequency range and count (:310-346)
    double fmax = 0.0, Sfmax = 0.0;
    for (int n = 0; n < nf; n++) { fmax = dmax(fmax, sp.f[n]); Sfmax = dmax(Sfmax, Sf[n]); }
    fmax = 2.0 * fmax;
    int ind1 = 0, ind2 = nf - 1;
    bool first = true;
    for (int n = 0; n < nf; n++)
        if (Sf[n] > Sfmax * w->sprdthr && sp.f[n] < fmax) {
            if (first) { ind1 = n; first = false; }
            ind2 = n;
        }
    int K = (int)std::ceil(p->rtlength * (sp.f[ind2] - sp.f[ind1]) + 1);
    K = (int)dmax(K * 1.0, 200.0);
    const double dfgen = (sp.f[ind2] - sp.f[ind1]) / K;
    std::vector<double> fgen(K), phigen(K), thgen(K), kgen(K), wgen(K), vargen(K), vargenq(K);
    for (int i = 0; i < K; i++) fgen[i] = sp.f[ind1] + i * dfgen;
    // ---- random phases, then directions from the CDF of the interpolated
    // directional distribution (:348-425)
    std::default_random_engine gen(w->seed);
    std::uniform_real_distribution<double> uni(0.0, 1.0);
    for (int i = 0; i < K; i++) phigen[i] = uni(gen) * 2.0 * PI_R;
    {
        std::vector<double> pdf(nd), cdf(nd);
        for (int i = 0; i < K; i++) {
            for (int d = 0; d < nd; d++)
                pdf[d] = interp_bilinear(nf, nd, sp.f.data(), sp.d.data(), sp.S.data(), fgen[i], sp.d[d]);
            double s = 0;
            for (int d = 0; d < nd; d++) s = s + pdf[d];
            for (int d = 0; d < nd; d++) pdf[d] = pdf[d] / s;
            cdf[0] = pdf[0];
            for (int d = 1; d < nd; d++) cdf[d] = cdf[d - 1] + 0.5 * (pdf[d - 1] + pdf[d]);
            const double u = uni(gen);
            thgen[i] = interp_search(nd, cdf.data(), sp.d.data(), u);
        }
    }
    // ---- wave numbers (Soulsby 2006, three Newton steps; :427-452)
    for (int i = 0; i < K; i++) {
        const double hh = w->offdepth;
        const double om = 2 * PI_R / ((1 / fgen[i]));
        const double x = om * om * hh / p->g;
        double y = std::sqrt(x) * (x < 1) + x * (x >= 1);
        for (int it = 0; it < 3; it++) {
            const double t = std::tanh(y);
            y = y - ((y * t - x) / (t + y * (1 - t * t)));
        }
        kgen[i] = y / hh;
        wgen[i] = om;
    }
    // ---- Trep (:458-472)
    {
        double a = 0.0, b = 0.0;
        for (int n = 0; n < nf; n++)
            if (Sf[n] >= Sfmax * 0.01) { a += (Sf[n] / dmax(sp.f[n], 0.001)); b += Sf[n]; }
        *Trep = (double)(float)(a / b);
    }
    // ---- internal time axis and tapers (:478-560)
    double dtin = p->dtbc;
    if (dtin > 0.5 / fgen[K - 1]) dtin = 0.5 / fgen[K - 1];
    int N = (int)(std::ceil(1 / dfgen / dtin) + 1);
    if ((std::ceil(N / 2.0f) - N / 2.0f) > 0) N = N + 1;
    if (N > 65535 || (double)(N - 1) * dtin < (tslenbc - 1) * p->dtbc) return XBG_ERR_ARG;
    std::vector<double> taperf(N, 1.0), taperw(N, 1.0);
    {
        const double Tbc = 1 / fgen[0];
        const int ntaper = (int)((5.0 * Tbc) / dtin);
        for (int n = 0; n < (int)dmin(1.0 * ntaper, 1.0 * N); n++) {
            taperf[n] = std::tanh(5.0 * n / ntaper);
            taperw[n] = std::tanh(5.0 * n / ntaper);
        }
        for (int n = N; n > 0; n--) {
            const double tn = (n - 1) * dtin;
            if (tn > (p->rtlength - ntaper * dtin)) taperf[n - 1] = std::tanh(5.0 * (p->rtlength - tn) / dtin / ntaper);
            if (tn > p->rtlength) taperf[n - 1] = 0;
        }
    }
    // ---- component variances (:565-591)
    double sumvar = 0.0;
    for (int i = 0; i < K; i++) {
        vargen[i] = interp_bilinear(nf, nd, sp.f.data(), sp.d.data(), sp.S.data(), fgen[i], thgen[i]);
        sumvar = sumvar + vargen[i];
    }
    const double scale = std::pow(Hm0 / (4.0 * std::sqrt(sumvar * dfgen)), 2);
    for (int i = 0; i < K; i++) vargen[i] = vargen[i] * scale;
    for (int i = 0; i < K; i++) vargenq[i] = dmin(vargen[i], interp_uniform(nf, sp.f.data(), Sf.data(), fgen[i]));
    // ---- Fourier indices, coefficients at the first offshore point, bins (:603-774)
    const int F0 = (int)std::floor(fgen[0] / dfgen);
    std::vector<int> F(K), bin(K);
    std::vector<double> ar(K), ai(K), sinth(K), argc(K + 1);
    const std::complex<double> iu(0.0, 1.0);
    for (int i = 0; i < K; i++) {
        F[i] = F0 + i;
        const std::complex<double> c = std::sqrt(2.0 * vargen[i] * dfgen) / 2 * std::exp(iu * phigen[i]);
        ar[i] = c.real(); ai[i] = c.imag();
        sinth[i] = std::sin(thgen[i]);
        argc[i + 1] = std::imag(std::log(std::conj(c)));
    }
    argc[0] = std::imag(std::log(std::conj(std::complex<double>(0.0, 0.0))));
    {
        std::vector<double> left(nbin), right(nbin);
        for (int b = 0; b < nbin; b++) {
            left[b] = std::fmod((b * p->dtheta + p->thetamin), 2 * PI_R);
            right[b] = std::fmod(((b + 1) * p->dtheta + p->thetamin), 2 * PI_R);
        }
        for (int i = 0; i < K; i++) {
            bin[i] = -1;
            for (int b = 0; b < nbin; b++) {
                const bool in = left[b] > right[b]
                                    ? ((thgen[i] >= left[b] && thgen[i] <= (2 * PI_R)) ||
                                       (thgen[i] >= 0.0 && thgen[i] <= right[b]))
                                    : (thgen[i] >= left[b] && thgen[i] <= right[b]);
                if (in) { bin[i] = b; break; }
            }
        }
        // components set to their bin centres (the bound waves see these; the
        // wave trains were laid out with the drawn directions)
        if (w->nspr == 1)
            for (int i = 0; i < K; i++)
                if (bin[i] > 0) thgen[i] = left[bin[i]] + p->dtheta * 0.5;
    }
    // components of each bin, in component order
    std::vector<int> order, bstart(nbin), bcount(nbin);
    for (int b = 0; b < nbin; b++) {
        bstart[b] = (int)order.size();
        for (int i = 0; i < K; i++)
            if (bin[i] == b) order.push_back(i);
        bcount[b] = (int)order.size() - bstart[b];
    }
    std::vector<int> Fo(order.size());
    std::vector<double> aro(order.size()), aio(order.size()), ko(order.size()), so(order.size());
    for (size_t c = 0; c < order.size(); c++) {
        const int i = order[c];
        Fo[c] = F[i]; aro[c] = ar[i]; aio[c] = ai[i]; ko[c] = kgen[i]; so[c] = sinth[i];
    }
    const int Kb = (int)order.size();
    // ---- device
    DevBufs B;
    int n2 = 1, logn = 0;
    while (n2 < N) { n2 <<= 1; logn++; }
    const std::vector<double2> Wn = twiddles(N), W2 = twiddles(n2);
    double2* dW = B.put(Wn);
    double2* dW2 = B.put(W2);
    double* dtw = B.put(taperw);
    double* dtf = B.put(taperf);
    int *dF = B.put(Fo), *dbs = B.put(bstart), *dbc = B.put(bcount);
    double *dar = B.put(aro), *dai = B.put(aio), *dk = B.put(ko), *ds = B.put(so);
    double2* dG = B.get<double2>((size_t)ny * (Kb > 0 ? Kb : 1));
    const int nblk = (N + WG_T - 1) / WG_T;
    double* deta = B.get<double>((size_t)ny * N);
    double* dpart = B.get<double>((size_t)ny * (nbin + 1) * nblk);
    double* dsd = B.get<double>((size_t)ny * (nbin + 1));
    double2* dX = B.get<double2>((size_t)ny * n2);
    double2* dY = B.get<double2>((size_t)ny * n2);
    double* damp = B.get<double>((size_t)ny * N);
    double* dSt = B.get<double>((size_t)tslenbc * nbin * ny);
    int* dbad = B.get<int>(1);
    std::vector<double> thv(thgen), argv(argc);
    double *dkg = B.put(kgen), *dwg = B.put(wgen), *dth = B.put(thv), *dfg = B.put(fgen), *dvq = B.put(vargenq),
           *darg = B.put(argv);
    Pair* dP = B.get<Pair>((size_t)(K - 1) * K);
    double4* dGq = B.get<double4>((size_t)ny * K);
    double* dq = B.get<double>((size_t)tslenbc * 4 * ny);
    if (!dW || !dW2 || !dtw || !dtf || !dF || !dbs || !dbc || !dar || !dai || !dk || !ds || !dG || !deta || !dpart ||
        !dsd || !dX || !dY || !damp || !dSt || !dbad || !dkg || !dwg || !dth || !dfg || !dvq || !darg || !dP ||
        !dGq || !dq)
        return XBG_ERR_NOMEM;
    cudaMemset(dbad, 0, sizeof(int));
    cudaMemset(dGq, 0, (size_t)ny * K * sizeof(double4));
    // wave trains and their envelope
    if (Kb > 0) k_wg_coef<<<dim3((Kb + 127) / 128, ny), 128>>>(dar, dai, dk, ds, Kb, ny, p->dx, dG);
    k_wg_zeta<<<dim3(nblk, ny), WG_T>>>(dG, dF, dbs, dbc, Kb, nbin, N, dW, dtw, deta, dpart);
    k_wg_std<<<(ny * (nbin + 1) + 255) / 256, 256>>>(dpart, nblk, nbin, ny, N, dsd);
    const size_t tot = (size_t)ny * n2;
    const unsigned gb = (unsigned)((tot + 255) / 256), gh = (unsigned)((tot / 2 + 255) / 256);
    k_wg_fft_load<<<gb, 256>>>(deta, N, n2, logn, ny, dX);
    for (int half = 1; half < n2; half <<= 1) k_wg_fft_stage<<<gh, 256>>>(dX, n2, half, ny, dW2, -1);
    k_wg_fft_hilbert<<<gb, 256>>>(dX, n2, logn, ny, dY);
    for (int half = 1; half < n2; half <<= 1) k_wg_fft_stage<<<gh, 256>>>(dY, n2, half, ny, dW2, +1);
    k_wg_fft_amp<<<(unsigned)(((size_t)ny * N + 255) / 256), 256>>>(dY, N, n2, ny, damp);
    const size_t nst = (size_t)tslenbc * nbin * ny;
    k_wg_st<<<(unsigned)((nst + 255) / 256), 256>>>(damp, dsd, nbin, ny, N, tslenbc, p->dtbc, dtin, p->rho, p->g,
                                                    p->dtheta, dSt, dbad);
    // bound long waves
    PairIn PI{dkg, dwg, dth, dfg, dvq, darg};
    if (K > 1) {
        k_wg_pairs<<<dim3((K + 127) / 128, K - 1), 128>>>(PI, K, dfgen, p->g, w->offdepth, w->nmax, w->fcutoff, dP);
        k_wg_bound<<<dim3((ny + 127) / 128, K - 1), 128>>>(dP, K, ny, p->dx, dGq);
    }
    k_wg_q<<<(unsigned)(((size_t)tslenbc * ny + 127) / 128), 128>>>(dGq, K, ny, N, dW, dtf, tslenbc, p->dtbc, dtin,
                                                                   dq);
    if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) return XBG_ERR_CUDA;
    int bad = 0;
    if (cudaMemcpy(&bad, dbad, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(St, dSt, nst * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(q, dq, (size_t)tslenbc * 4 * ny * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)
        return XBG_ERR_CUDA;
    return bad ? XBG_ERR_NAN : XBG_OK;
}

extern "C" int xbg_gen_constant_waves(const xbg_params* p, const double* rec, int n, const double* theta,
                                      double* St, double* q, double* Tp) {
    if (!p || !rec || n < 1 || !theta || !St || !q || !Tp) return XBG_ERR_ARG;
    const int ny = p->ny, nt = p->ntheta;
    std::vector<double> sc(nt);
    for (int r = 0; r < n; r++) {
        const double Hs = rec[5 * r + 1], Dp = rec[5 * r + 3], s = rec[5 * r + 4];
        Tp[r] = rec[5 * r + 2];
        const double eetot = Hs * Hs * p->rho * p->g / (16.0 * p->dtheta);
        for (int j = 0; j < ny; j++)
            for (int c = 0; c < 4; c++) q[j + c * ny + (size_t)r * ny * 4] = 0.0;
        double sumcos = 0.0;
        for (int t = 0; t < nt; t++) {
            sc[t] = std::pow(std::cos((theta[t] - Dp) / 2.0), 2.0 * s);
            sumcos = sumcos + sc[t];
        }
        for (int t = 0; t < nt; t++) {
            const double v = sc[t] / sumcos * eetot;
            for (int j = 0; j < ny; j++) St[j + t * ny + (size_t)r * ny * nt] = v;
        }
    }
    return XBG_OK;
}
