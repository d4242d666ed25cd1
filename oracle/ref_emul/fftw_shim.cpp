// TEST INFRASTRUCTURE ONLY: the FFTW entry points the reference's wave-group
// generator calls (makjonswap.cpp, tools.cpp), as an exact O(N^2) discrete
// Fourier transform in double with FFTW's sign convention and without
// normalisation.  The twiddle angle 2 pi ((k n) mod N) / N is reduced
// exactly in integers before the cosine and sine, so the transform is
// accurate to a few ulps; FFTW computes the same transform to rounding.
#include <cmath>
#include <cstdlib>
#include <vector>

#include "fftw3.h"

struct fftw_plan_s {
    int n, sign;
    fftw_complex *in, *out;
    std::vector<double> c, s;   // cos, sin of 2 pi m / n
};

extern "C" {

void* fftw_malloc(size_t n) { return std::malloc(n); }
void fftw_free(void* p) { std::free(p); }

fftw_plan fftw_plan_dft_1d(int n, fftw_complex* in, fftw_complex* out, int sign, unsigned) {
    fftw_plan p = new fftw_plan_s();
    p->n = n; p->sign = sign; p->in = in; p->out = out;
    p->c.resize(n); p->s.resize(n);
    const long double tp = 6.283185307179586476925286766559L;
    for (int m = 0; m < n; m++) {
        long double a = tp * (long double)m / (long double)n;
        p->c[m] = (double)cosl(a);
        p->s[m] = (double)sinl(a);
    }
    return p;
}

void fftw_execute(const fftw_plan p) {
    const int n = p->n;
    std::vector<double> re(n), im(n);
    for (int k = 0; k < n; k++) {
        double sr = 0.0, si = 0.0;
        for (int m = 0; m < n; m++) {
            const double xr = p->in[m][0], xi = p->in[m][1];
            if (xr == 0.0 && xi == 0.0) continue;
            const int idx = (int)(((long long)k * m) % n);
            const double c = p->c[idx], s = p->sign * p->s[idx];
            sr += xr * c - xi * s;
            si += xr * s + xi * c;
        }
        re[k] = sr; im[k] = si;
    }
    for (int k = 0; k < n; k++) { p->out[k][0] = re[k]; p->out[k][1] = im[k]; }
}

void fftw_destroy_plan(fftw_plan p) { delete p; }

}  // extern "C"
