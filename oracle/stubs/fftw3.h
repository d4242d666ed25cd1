/* Stub for building the reference CPU sources in place: only the FFTW type
 * names that XBeachGPU.h mentions.  FFTW itself is not installed and is not
 * on the step path.  TEST INFRASTRUCTURE ONLY. */
#ifndef XBG_FFTW3_STUB_H
#define XBG_FFTW3_STUB_H
typedef double fftw_complex[2];
typedef struct fftw_plan_s* fftw_plan;
#endif
