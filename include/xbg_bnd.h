/*
 * xbg_bnd.h -- offshore wave-boundary synthesis of the B200-native XBeach_GPU
 * step: the records St (wave energy per directional bin along the offshore
 * boundary) and qbnd (bound long-wave fluxes) that xbg_set_wave_boundary
 * takes, generated from a JONSWAP record as the reference's makjonswap +
 * GenWGnLBW do (makjonswap.cpp:73-1419, called at Wavestep.cu:142-146 and
 * :553), or from constant-wave records as GenCstWave does
 * (makjonswap.cpp:24-71).
 *
 * The wave-group generator's heavy parts run on the current CUDA device in
 * double precision: the wave-train synthesis along the boundary (one inverse
 * Fourier sum per offshore point and directional bin), the Hilbert envelope
 * (a radix-2 FFT per offshore point), the difference-interaction
 * coefficients of all component pairs and the bound long-wave sums.  The
 * serial set-up (spectrum, component frequencies, random phases and
 * directions drawn with std::default_random_engine as the reference does,
 * variances, binning) runs on the host.
 */
#ifndef XBG_BND_H
#define XBG_BND_H

#include "xbg.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct xbg_wavegen {
    double Hs, Tp;      /* significant height [m], peak period [s]            */
    double Dp;          /* mean direction [rad] relative to the grid, as
                           ReadJSWPBnd converts it (1.5 pi - grdalpha - Dp_deg
                           pi/180)                                            */
    double s, gamma;    /* directional spreading, peak enhancement            */
    double sprdthr;     /* spectral threshold of the component range (0.08)   */
    double offdepth;    /* water depth at the offshore boundary [m] (the
                           reference takes hh at ix = 0, iy = ny/2)           */
    double nmax;        /* cap on the bound-wave group-velocity ratio (0.8)  */
    double fcutoff;     /* lowest bound-wave difference frequency [Hz] (0)    */
    int    nspr;        /* 1: components at their bin centre directions (0)   */
    unsigned seed;      /* seed of the phase and direction draws; the
                           reference uses 0 (or the clock when random = 1)    */
} xbg_wavegen;

void xbg_wavegen_default(xbg_wavegen* w);

/* makjonswap + GenWGnLBW for one record w on the grid of p (ny, dx, ntheta,
 * thetamin, dtheta, dtbc, rtlength, rho, g): St[nrec][ntheta][ny] and
 * q[nrec][4][ny] host arrays with nrec = ceil(rtlength/dtbc) + 1 records
 * dtbc apart, and the representative period Trep (float-rounded, as the
 * reference's).  Allocates and frees its device buffers; synchronous. */
int xbg_gen_wave_groups(const xbg_params* p, const xbg_wavegen* w, double* St, double* q, int nrec,
                        double* Trep);

/* GenCstWave for n constant-wave records rec[k] = (time, Hs, Tp, Dp, s):
 * St[n][ntheta][ny] with the energy Hs^2 rho g / (16 dtheta) spread over the
 * bins as cos((theta - Dp)/2)^(2 s), q[n][4][ny] = 0, Tp[n].  theta: the
 * ntheta bin directions [rad].  Host only. */
int xbg_gen_constant_waves(const xbg_params* p, const double* rec, int n, const double* theta, double* St,
                           double* q, double* Tp);

#ifdef __cplusplus
}
#endif
#endif
