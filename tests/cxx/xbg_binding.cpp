// The binding a maintainer adds to the reference's host code: the device
// allocations of main and the body of mainloopGPU (Wave_gpu.cu:610-931) are
// replaced by one handle of libxbg_b200.so.  The reference keeps its
// parameter parsing (read_input.cpp), its boundary generation
// (makjonswap/GenWGnLBW, here the callback next_chunk) and its output
// variable list.  This file is compiled and run by the tests; the
// integration guide shows it verbatim.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "xbg.h"
#include "xbg_io.h"
#include "ref_host_types.h"   // in the reference's tree: #include "XBeachGPU.h"

static xbg_params to_xbg(const XBGPUParam& P) {
    xbg_params p;
    xbg_params_default(&p);
    p.nx = P.nx; p.ny = P.ny; p.dx = P.dx;
    p.swave = P.swave; p.flow = P.flow; p.sedtrans = P.sedtrans; p.morphology = P.morphology;
    p.g = P.g; p.rho = P.rho; p.eps = P.eps; p.cf = P.cf; p.cfsand = P.cfsand; p.cfreef = P.cfreef;
    p.nuh = P.nuh; p.nuhfac = P.nuhfac; p.usesmago = P.usesmago; p.smag = P.smag;
    p.lat = P.lat; p.fc = P.fc; p.Cd = P.Cd;
    p.wci = P.wci; p.hwci = P.hwci; p.breakmodel = P.breakmodel; p.gammaa = P.gammaa;
    p.n = P.n; p.alpha = P.alpha; p.gammax = P.gammax; p.beta = P.beta; p.fw = P.fw;
    p.fwsand = P.fwsand; p.fwreef = P.fwreef;
    p.roller = P.roller; p.thetamin = P.thetamin; p.thetamax = P.thetamax; p.dtheta = P.dtheta;
    p.D50 = P.D50; p.D90 = P.D90; p.rhosed = P.rhosed; p.wws = P.wws;
    p.drydzmax = P.drydzmax; p.wetdzmax = P.wetdzmax; p.maxslpchg = P.maxslpchg; p.por = P.por;
    p.morfac = P.morfac; p.sus = P.sus; p.bed = P.bed; p.facsk = P.facsk; p.facas = P.facas;
    p.wavebndtype = P.wavebndtype; p.CFL = P.CFL; p.sedstart = P.sedstart;
    p.outputtimestep = P.outputtimestep; p.endtime = P.endtime; p.dtbc = P.dtbc;
    p.rtlength = P.rtlength;
    return p;
}

// the reference's CUDA_CHECK exits on an error (Wavestep.cu:4-18); so does this
#define XBG_CHECK(x) do { int s_ = (x); if (s_ != XBG_OK) { \
    fprintf(stderr, "%s: %s\n", #x, xbg_status_string(s_)); exit(EXIT_FAILURE); } } while (0)

// One wave-boundary chunk as GenWGnLBW writes it (makjonswap.cpp:235):
// Stfile[nrec][ntheta][ny], qfile[nrec][4][ny] and Trep, for records
// t0 + m*dtbc.
struct WaveChunk { std::vector<double> St, q; int nrec; double t0; double Trep; };
typedef WaveChunk (*NextChunk)(const XBGPUParam& P, int ntheta, double t0, void* user);

// field id of an output variable name of Param.outvars
static int field_id(const std::string& name) {
    static const char* names[XBG_F_COUNT] = {
        "zb", "zs", "hh", "uu", "vv", "hu", "hv", "hum", "hvm", "qx", "qy", "ueu", "vev", "vmageu", "vmagev",
        "vu", "uv", "uuold", "vvold", "zsold", "dzsdt", "H", "E", "D", "DR", "R", "k", "c", "cg", "Fx", "Fy",
        "urms", "ust", "thetamean", "cfm", "fwm", "C", "ceqsg", "stdep", "dzb", "rolthick", "kturb", "Hmean",
        "uumean", "vvmean", "hhmean", "zsmean", "Cmean", "zsmax", "wetu", "wetv", "umeanbnd", "ee", "rr"};
    for (int k = 0; k < XBG_F_COUNT; k++)
        if (name == names[k]) return k;
    return -1;
}

// replaces the device allocations of main and the body of mainloopGPU;
// returns the number of coupled steps taken
long long mainloop_xbg(const XBGPUParam& Param, const std::vector<SLBnd>& slbnd,
                       const std::vector<WindBnd>& wndbnd, const float* zb_host,
                       NextChunk next_chunk, void* user) {
    xbg_params p = to_xbg(Param);
    XBG_CHECK(xbg_params_sanity(&p, std::min(slbnd.back().time, wndbnd.back().time)));
    xbg_handle* h = nullptr;
    XBG_CHECK(xbg_create(&p, XBG_FP32, &h));
    // sea level and wind series (flowbnd's inputs), as arrays
    std::vector<double> ts, w0, w1, tw, wu, wv;
    for (const SLBnd& s : slbnd) { ts.push_back(s.time); w0.push_back(s.wlev0); w1.push_back(s.wlev1); }
    for (const WindBnd& w : wndbnd) { tw.push_back(w.time); wu.push_back(w.U); wv.push_back(w.V); }
    XBG_CHECK(xbg_set_sealevel(h, ts.data(), w0.data(), w1.data(), (int)ts.size()));
    XBG_CHECK(xbg_set_wind(h, tw.data(), wu.data(), wv.data(), (int)tw.size()));
    // the first two wave-boundary chunks, [0, rtlength) in use and the next one
    // queued, before the initial state (whose offshore column comes from the
    // first record); slot 1 is always the queued chunk
    double next_t0 = 0.0;
    for (int slot = 0; slot < 2; slot++) {
        WaveChunk ch = next_chunk(Param, p.ntheta, next_t0, user);
        XBG_CHECK(xbg_set_wave_boundary(h, slot, ch.St.data(), ch.q.data(), ch.nrec, nullptr, ch.t0,
                                        ch.t0 + Param.rtlength, ch.Trep));
        next_t0 += Param.rtlength;
    }
    XBG_CHECK(xbg_init_state(h, zb_host, slbnd[0].wlev0, slbnd[0].wlev1));
    // map output in place of creatncfileUD + defncvar (Wave_gpu.cu:2943-2951):
    // Param.outvars, 3 dimensions or 4 for ee/rr; record 0 is the initial state
    const int nout = (int)Param.outvars.size();
    std::vector<int> ids(nout), ndims(nout);
    std::vector<const char*> names(nout);
    std::vector<std::vector<float>> host(nout);
    std::vector<void*> hp(nout);
    std::vector<const float*> hc(nout);
    for (int k = 0; k < nout; k++) {
        ids[k] = field_id(Param.outvars[k]);
        if (ids[k] < 0 || ids[k] == XBG_F_WETU || ids[k] == XBG_F_WETV || ids[k] == XBG_F_UMEANBND) {
            fprintf(stderr, "no map output for %s\n", Param.outvars[k].c_str());
            exit(EXIT_FAILURE);
        }
        size_t cnt = 0;
        XBG_CHECK(xbg_field_count(h, ids[k], &cnt));
        ndims[k] = (ids[k] == XBG_F_EE || ids[k] == XBG_F_RR) ? 4 : 3;
        names[k] = Param.outvars[k].c_str();
        host[k].resize(cnt);
        hp[k] = host[k].data();
        hc[k] = host[k].data();
    }
    xbg_nc* nc = nullptr;
    XBG_CHECK(xbg_nc_create(Param.outfile.c_str(), 1, p.nx, p.ny, p.dx, p.ntheta, p.dtheta, p.thetamin, nout,
                            names.data(), ndims.data(), &nc));
    XBG_CHECK(xbg_fetch_fields(h, ids.data(), nout, hp.data()));
    XBG_CHECK(xbg_sync(h));
    XBG_CHECK(xbg_nc_write_record(nc, 0.0, hc.data()));
    long long steps = 0;
    for (;;) {
        XBG_CHECK(xbg_advance(h, 64));            // up to 64 coupled steps, no host round trip
        double t, dt;
        int64_t nstep;
        int flags;
        XBG_CHECK(xbg_get_time(h, &t, &dt, &nstep, &flags));
        steps = nstep;
        if (flags & XBG_FLAG_NEED_BOUNDARY) {
            // the queued chunk went into use: generate and queue the one after it
            WaveChunk nx = next_chunk(Param, p.ntheta, next_t0, user);
            XBG_CHECK(xbg_set_wave_boundary(h, 1, nx.St.data(), nx.q.data(), nx.nrec, nullptr, nx.t0,
                                            nx.t0 + Param.rtlength, nx.Trep));
            next_t0 += Param.rtlength;
        }
        if (flags & XBG_FLAG_OUTPUT_DUE) {
            XBG_CHECK(xbg_output_done(h));        // means /= nstep, next output time
            // writenctimestep + the copy/writencvarstep loop (Wave_gpu.cu:819-832)
            XBG_CHECK(xbg_fetch_fields(h, ids.data(), nout, hp.data()));
            XBG_CHECK(xbg_sync(h));
            XBG_CHECK(xbg_nc_write_record(nc, t, hc.data()));
            XBG_CHECK(xbg_reset_means(h));
        }
        if (flags & XBG_FLAG_ENDED) break;
    }
    XBG_CHECK(xbg_nc_close(nc));
    XBG_CHECK(xbg_destroy(h));
    return steps;
}
