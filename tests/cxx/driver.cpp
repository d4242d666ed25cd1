// Test driver of the reference-side binding (xbg_binding.cpp): the
// reference's CPU-runnable case (linear beach, 200 x 100 cells of 5 m,
// 10 bins of 10 deg, Hm0 1.5 m, Tp 10 s, morfac 1) run through
// mainloop_xbg for a short time with map output.
//
//   driver <zb.f32> <St.f64> <q.f64> <nrec> <endtime> <outputtimestep> <out.nc>
//
// zb: nx*ny floats; St, q: one boundary chunk (nrec records, dtbc = 1 s) that
// every call of the chunk callback hands out again.  Prints "steps=N".
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "xbg.h"
#include "ref_host_types.h"

struct WaveChunk { std::vector<double> St, q; int nrec; double t0; double Trep; };
typedef WaveChunk (*NextChunk)(const XBGPUParam& P, int ntheta, double t0, void* user);
long long mainloop_xbg(const XBGPUParam& Param, const std::vector<SLBnd>& slbnd,
                       const std::vector<WindBnd>& wndbnd, const float* zb_host,
                       NextChunk next_chunk, void* user);

struct Inputs { std::vector<double> St, q; int nrec; };

static WaveChunk same_chunk(const XBGPUParam&, int, double t0, void* user) {
    const Inputs* in = static_cast<const Inputs*>(user);
    return WaveChunk{in->St, in->q, in->nrec, t0, 10.0 / 1.1};
}

template <class T>
static std::vector<T> read_all(const char* path, size_t n) {
    std::vector<T> v(n);
    FILE* f = fopen(path, "rb");
    if (!f || fread(v.data(), sizeof(T), n, f) != n) {
        fprintf(stderr, "cannot read %zu values from %s\n", n, path);
        exit(EXIT_FAILURE);
    }
    fclose(f);
    return v;
}

int main(int argc, char** argv) {
    if (argc != 8) {
        fprintf(stderr, "usage: driver zb.f32 St.f64 q.f64 nrec endtime outputtimestep out.nc\n");
        return 2;
    }
    XBGPUParam P;
    P.nx = 200; P.ny = 100; P.dx = 5.0;
    P.thetamin = -50 * 3.14159265 / 180; P.thetamax = 50 * 3.14159265 / 180; P.dtheta = 10 * 3.14159265 / 180;
    P.D50 = 0.0002; P.D90 = 0.0003; P.morfac = 1.0;
    P.wavebndtype = 4; P.sedtrans = 1; P.morphology = 1; P.sedstart = 0.0;
    P.CFL = 0.7; P.eps = 0.01; P.dtbc = 1.0; P.rtlength = 3600.0;
    P.endtime = atof(argv[5]);
    P.outputtimestep = atof(argv[6]);
    P.outfile = argv[7];
    P.outvars = {"zb", "zs", "uu", "vv", "H", "hh", "C", "Hmean", "ee"};
    const int nt = 10;
    Inputs in;
    in.nrec = atoi(argv[4]);
    std::vector<float> zb = read_all<float>(argv[1], (size_t)P.nx * P.ny);
    in.St = read_all<double>(argv[2], (size_t)in.nrec * nt * P.ny);
    in.q = read_all<double>(argv[3], (size_t)in.nrec * 4 * P.ny);
    std::vector<SLBnd> sl = {{0.0, 0.0, 0.0}, {1e6, 0.0, 0.0}};
    std::vector<WindBnd> wnd = {{0.0, 0.0, 0.0, 0.0, 0.0, 0.0}, {1e6, 0.0, 0.0, 0.0, 0.0, 0.0}};
    long long steps = mainloop_xbg(P, sl, wnd, zb.data(), same_chunk, &in);
    printf("steps=%lld\n", steps);
    return 0;
}
