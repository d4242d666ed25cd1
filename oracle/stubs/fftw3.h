/* Stub for building the reference CPU sources in place: the FFTW names the
 * reference uses.  FFTW itself is not installed; ref_emul/fftw_shim.cpp
 * implements these few entry points as an exact discrete Fourier transform
 * with FFTW's conventions (FFTW_FORWARD: exponent -2 pi i k n / N,
 * FFTW_BACKWARD: +2 pi i k n / N, no normalisation).  TEST INFRASTRUCTURE
 * ONLY. */
#ifndef XBG_FFTW3_STUB_H
#define XBG_FFTW3_STUB_H
#include <stddef.h>
typedef double fftw_complex[2];
typedef struct fftw_plan_s* fftw_plan;
#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_ESTIMATE (1U << 6)
#ifdef __cplusplus
extern "C" {
#endif
void* fftw_malloc(size_t n);
void fftw_free(void* p);
fftw_plan fftw_plan_dft_1d(int n, fftw_complex* in, fftw_complex* out, int sign, unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);
#ifdef __cplusplus
}
#endif
#endif
