// TEST INFRASTRUCTURE ONLY: plain-C entry points onto the reference's wave
// boundary generators (makjonswap.cpp: makjonswap + GenWGnLBW, GenCstWave),
// compiled in place from the reference checkout with the FFTW shim, so the
// tests can compare the library's generator with them.  Nothing is restated.
#include <cmath>
#include <vector>

#include "XBeachGPU.h"

template <class T> const T& min(const T& a, const T& b) { return !(b < a) ? a : b; }
template <class T> const T& max(const T& a, const T& b) { return (a < b) ? b : a; }
template const double& min<double>(const double&, const double&);
template const double& max<double>(const double&, const double&);

void write_text_to_log_file(std::string) {}

void makjonswap(XBGPUParam Param, std::vector<Wavebndparam> wavebnd, int step, int& nfreq, int& ntheta,
                double*& HRfreq, double*& HRdir, double*& HRSpec);
void GenWGnLBW(XBGPUParam Param, int nf, int ndir, double* HRfreq, double* HRdir, double* HRSpec, float& Trep,
               double*& qfile, double*& Stfile);
void GenCstWave(XBGPUParam Param, std::vector<Wavebndparam> wavebnd, float* theta, double*& Stfile,
                double*& qfile, double*& Tpfile);

extern "C" {

// p: ny, ntheta, random, nspr (ints) and dx, thetamin, dtheta, dtbc, rtlength,
// rho, g, sprdthr, offdepth, nmax, fcutoff (doubles); w: Hs, Tp, Dp, s, gamma.
// St: ny*ntheta*(ceil(rtlength/dtbc)+1), q: 4*ny*(same).
void ref_wavegen(const int* pi_, const double* pd, const double* w, double* St, double* q, double* Trep) {
    XBGPUParam P;
    P.ny = pi_[0]; P.ntheta = pi_[1]; P.random = pi_[2]; P.nspr = pi_[3];
    P.dx = pd[0]; P.thetamin = pd[1]; P.dtheta = pd[2]; P.dtbc = pd[3]; P.rtlength = pd[4];
    P.rho = pd[5]; P.g = pd[6]; P.sprdthr = pd[7]; P.offdepth = pd[8]; P.nmax = pd[9]; P.fcutoff = pd[10];
    Wavebndparam b;
    b.time = 0.0; b.Hs = w[0]; b.Tp = w[1]; b.Dp = w[2]; b.s = w[3]; b.gamma = w[4];
    std::vector<Wavebndparam> v(1, b);
    int nf = 0, nd = 0;
    double *f = nullptr, *d = nullptr, *S = nullptr;
    makjonswap(P, v, 0, nf, nd, f, d, S);
    float tr = 0.0f;
    GenWGnLBW(P, nf, nd, f, d, S, tr, q, St);
    *Trep = tr;
    free(f); free(d); free(S);
}

// the JONSWAP spectrum alone: nf x nd values HRSpec[f + d*nf] into S (cap
// values), the axes into f / d; returns nf * nd
int ref_jonswap(const double* w, double* fo, double* dout, double* So, int cap) {
    XBGPUParam P;
    Wavebndparam b;
    b.Hs = w[0]; b.Tp = w[1]; b.Dp = w[2]; b.s = w[3]; b.gamma = w[4];
    std::vector<Wavebndparam> v(1, b);
    int nf = 0, nd = 0;
    double *f = nullptr, *d = nullptr, *S = nullptr;
    makjonswap(P, v, 0, nf, nd, f, d, S);
    if (nf * nd <= cap) {
        for (int k = 0; k < nf; k++) fo[k] = f[k];
        for (int k = 0; k < nd; k++) dout[k] = d[k];
        for (int k = 0; k < nf * nd; k++) So[k] = S[k];
    }
    free(f); free(d); free(S);
    return nf * nd;
}

// GenCstWave for n records (time, Hs, Tp, Dp, s per record in rec)
void ref_gencst(const int* pi_, const double* pd, const double* rec, int n, const float* theta, double* St,
                double* q, double* Tp) {
    XBGPUParam P;
    P.ny = pi_[0]; P.ntheta = pi_[1];
    P.dtheta = pd[2]; P.rho = pd[5]; P.g = pd[6];
    std::vector<Wavebndparam> v(n);
    for (int k = 0; k < n; k++) {
        v[k].time = rec[5 * k]; v[k].Hs = rec[5 * k + 1]; v[k].Tp = rec[5 * k + 2];
        v[k].Dp = rec[5 * k + 3]; v[k].s = rec[5 * k + 4];
    }
    GenCstWave(P, v, const_cast<float*>(theta), St, q, Tp);
}

}  // extern "C"
