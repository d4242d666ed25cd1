/*
 * ref_kernels.cpp -- TEST INFRASTRUCTURE ONLY.
 *
 * Runs the reference's own CUDA kernels (Wave_kernel.cu, Flow_kernel.cu,
 * Sediment_kernel.cu, compiled in place as host C++ through cuda_emul.h) in
 * the launch order of the reference host functions:
 *   ubnd1D           flowbnd,      Wave_gpu.cu:1063-1073
 *   flow kernels     flowstep,     Wave_gpu.cu:1142-1397
 *   sediment kernels sedimentstep, Wave_gpu.cu:1462-1606
 * Launches are serial (iy outer, ix inner, one thread per block) over exactly
 * nx x ny threads, so no thread runs outside the grid.  Two launches differ
 * from a plain serial run and are documented where they happen:
 *   - ubnd1D is run with every thread reading the pre-kernel uu column (the
 *     GPU version races on it, Flow_kernel.cu:207-212);
 *   - vdvdy_fixbnd is not run: it stores an uninitialised local into every
 *     cell (Flow_kernel.cu:1076-1100); the only row it is meant to change
 *     (iy = ny-1) is never read by eulervstep.
 */
#include "cuda_emul.h"
#include "ref_driver.h"
#include <vector>

dim3 threadIdx, blockIdx, blockDim, gridDim;

using DECNUM = float;
#include "Wave_kernel.cu"
#include "Flow_kernel.cu"
#include "Sediment_kernel.cu"

namespace {
template <class K>
void launch(int nx, int ny, K k) {
    blockDim = {1, 1, 1};
    gridDim = {(unsigned)nx, (unsigned)ny, 1};
    threadIdx = {0, 0, 0};
    for (int by = 0; by < ny; by++)
        for (int bx = 0; bx < nx; bx++) {
            blockIdx = {(unsigned)bx, (unsigned)by, 0};
            k();
        }
}
}  // namespace

void ref_flow_boundary(RefState& s) {
    int nx = s.nx, ny = s.ny;
    float* uu = s.f(XBG_F_UU);
    std::vector<float> col0(ny), outu(ny);
    for (int iy = 0; iy < ny; iy++) col0[iy] = uu[iy * nx];
    /* one thread per row, each seeing the pre-kernel uu column */
    blockDim = {1, 1, 1};
    gridDim = {(unsigned)nx, (unsigned)ny, 1};
    threadIdx = {0, 0, 0};
    for (int by = 0; by < ny; by++) {
        for (int iy = 0; iy < ny; iy++) uu[iy * nx] = col0[iy];
        blockIdx = {0, (unsigned)by, 0};
        if (s.P.swave == 1)
            ubnd1D(nx, ny, s.P.dx, s.dt, s.P.g, s.P.rho, (float)s.totaltime, s.timesincelast, s.timenext,
                   s.zsbndi, s.zsbndn, s.Trep, s.qbndold.data(), s.qbndnew.data(), s.f(XBG_F_ZS), uu,
                   s.f(XBG_F_VV), s.f(XBG_F_VU), s.f(XBG_F_UMEANBND), s.vmeanbnd.data(), s.f(XBG_F_ZB),
                   s.f(XBG_F_CG), s.f(XBG_F_HUM), s.f(XBG_F_CFM), s.f(XBG_F_FX), s.f(XBG_F_HH));
        else
            ubnd1Dnowaves(nx, ny, s.P.dx, s.dt, s.P.g, s.P.rho, (float)s.totaltime, s.timesincelast,
                          s.timenext, s.zsbndi, s.zsbndn, s.f(XBG_F_ZS), uu, s.f(XBG_F_VV), s.f(XBG_F_VU),
                          s.f(XBG_F_UMEANBND), s.vmeanbnd.data(), s.f(XBG_F_ZB), s.f(XBG_F_HUM),
                          s.f(XBG_F_CFM), s.f(XBG_F_HH));
        outu[by] = uu[by * nx];
    }
    for (int iy = 0; iy < ny; iy++) uu[iy * nx] = outu[iy];
}

void ref_flow_step(RefState& s) {
    int nx = s.nx, ny = s.ny;
    xbg_params& P = s.P;
    float dx = P.dx, dt = s.dt, eps = P.eps, uumin = 0.0f;
    float *zs = s.f(XBG_F_ZS), *zb = s.f(XBG_F_ZB), *hh = s.f(XBG_F_HH), *uu = s.f(XBG_F_UU),
          *vv = s.f(XBG_F_VV), *hu = s.f(XBG_F_HU), *hv = s.f(XBG_F_HV), *hum = s.f(XBG_F_HUM),
          *hvm = s.f(XBG_F_HVM), *qx = s.f(XBG_F_QX), *qy = s.f(XBG_F_QY), *uuold = s.f(XBG_F_UUOLD),
          *vvold = s.f(XBG_F_VVOLD), *zsold = s.f(XBG_F_ZSOLD), *DR = s.f(XBG_F_DR), *cfm = s.f(XBG_F_CFM),
          *urms = s.f(XBG_F_URMS), *Fx = s.f(XBG_F_FX), *Fy = s.f(XBG_F_FY), *vu = s.f(XBG_F_VU),
          *uv = s.f(XBG_F_UV), *ueu = s.f(XBG_F_UEU), *vev = s.f(XBG_F_VEV), *vmageu = s.f(XBG_F_VMAGEU),
          *vmagev = s.f(XBG_F_VMAGEV), *dzsdt = s.f(XBG_F_DZSDT), *ust = s.f(XBG_F_UST),
          *thetamean = s.f(XBG_F_THETAMEAN);
    int *wetu = s.wetu.data(), *wetv = s.wetv.data();
    float *dzsdx = s.dzsdx.data(), *dzsdy = s.dzsdy.data(), *ududx = s.ududx.data(), *vdudy = s.vdudy.data(),
          *udvdx = s.udvdx.data(), *vdvdy = s.vdvdy.data(), *nuh = s.nuh.data(), *viscu = s.viscu.data(),
          *viscv = s.viscv.data();
    float windu = s.windu, windv = s.windv;
    launch(nx, ny, [&] { wlevslopes(nx, ny, dx, eps, zs, dzsdx, dzsdy, hh); });
    launch(nx, ny, [&] { udepthmomcont(nx, ny, dx, eps, uumin, wetu, zs, uu, hh, hum, hu, zb); });
    launch(nx, ny, [&] { vdepthmomcont(nx, ny, dx, eps, uumin, wetv, zs, vv, hh, hvm, hv, zb); });
    launch(nx, ny, [&] { ududx_adv(nx, ny, dx, hu, hum, uu, ududx); });
    launch(nx, ny, [&] { vdudy_adv(nx, ny, dx, hv, hum, uu, vv, vdudy); });
    launch(nx, ny, [&] { smago(nx, ny, dx, P.rho, P.nuhfac, hh, uu, vv, P.nuh, nuh, DR, P.usesmago); });
    launch(nx, ny, [&] { viscou1(nx, ny, dx, P.rho, eps, P.nuhfac, nuh, hh, hum, hvm, DR, uu, wetu, viscu); });
    launch(nx, ny, [&] { viscou2(nx, ny, dx, P.rho, eps, P.nuhfac, nuh, hh, hum, hvm, DR, uu, wetu, viscu); });
    launch(nx, ny, [&] { eulerustep(nx, ny, dx, dt, P.g, P.rho, cfm, P.fc, windu, P.Cd, uu, urms, ududx, vdudy, viscu, dzsdx, hu, hum, Fx, vu, ueu, vmageu, wetu); });
    launch(nx, ny, [&] { latbnd(nx, ny, uu); });
    launch(nx, ny, [&] { vdvdy_adv(nx, ny, dx, hv, hvm, vv, vdvdy); });
    /* vdvdy_fixbnd: not run, see the file header */
    launch(nx, ny, [&] { udvdx_adv(nx, ny, dx, hu, hvm, uu, vv, udvdx); });
    launch(nx, ny, [&] { viscov1(nx, ny, dx, P.rho, eps, P.nuhfac, nuh, hh, hum, hvm, DR, vv, wetv, viscv); });
    launch(nx, ny, [&] { viscovbnd(nx, ny, viscv); });
    launch(nx, ny, [&] { viscov2(nx, ny, dx, P.rho, eps, P.nuhfac, nuh, hh, hum, hvm, DR, vv, wetv, viscv); });
    launch(nx, ny, [&] { eulervstep(nx, ny, dx, dt, P.g, P.rho, cfm, P.fc, windv, P.Cd, vv, urms, udvdx, vdvdy, viscv, dzsdy, hv, hvm, Fy, uv, vev, vmagev, wetv); });
    launch(nx, ny, [&] { vvlatbnd(nx, ny, vv); });
    /* viscu / viscv are reused as wrk1 / wrk2, Wave_gpu.cu:1281 */
    launch(nx, ny, [&] { wrkuu2Ocorr(nx, ny, dx, dt, eps, uu, uuold, hum, zs, zb, qx, qy, viscu, viscv); });
    launch(nx, ny, [&] { uu2Ocorr(nx, ny, dx, dt, uu, uuold, hum, qx, qy, viscu, viscv); });
    launch(nx, ny, [&] { wrkvv2Ocorr(nx, ny, dx, dt, eps, vv, vvold, hvm, zs, zb, qx, qy, viscu, viscv); });
    launch(nx, ny, [&] { vv2Ocorr(nx, ny, dx, dt, vv, vvold, hvm, qx, qy, viscu, viscv); });
    launch(nx, ny, [&] { depthhu(nx, ny, dx, uumin, eps, hh, uu, hu, zs, zb); });
    launch(nx, ny, [&] { depthhv(nx, ny, dx, uumin, eps, hh, vv, hv, zs, zb); });
    launch(nx, ny, [&] { CalcQFlow(nx, ny, uu, hu, vv, hv, qx, qy); });
    launch(nx, ny, [&] { continuity(nx, ny, dx, dt, eps, qx, qy, zs, hh, zb, dzsdt); });
    launch(nx, ny, [&] { wrkzs2Ocorr(nx, ny, dx, dt, eps, zs, zsold, uu, vv, zb, viscu, viscv); });
    launch(nx, ny, [&] { zs2Ocorr(nx, ny, dx, dt, zs, qx, qy, viscu, viscv); });
    launch(nx, ny, [&] { latbnd(nx, ny, zs); });
    launch(nx, ny, [&] { hsbnd(nx, ny, eps, hh, zb, zs); });
    launch(nx, ny, [&] { calcuvvu(nx, ny, dx, uu, vv, vu, uv, ust, thetamean, ueu, vev, vmageu, vmagev, uuold, vvold, zs, zsold, wetu, wetv); });
    launch(nx, ny, [&] { uvlatbnd(nx, ny, vu, uv, ueu, vev, vmageu, vmagev); });
}

void ref_sediment_step(RefState& s) {
    int nx = s.nx, ny = s.ny;
    xbg_params& P = s.P;
    float dx = P.dx, dt = s.dt, eps = P.eps, Trep = s.Trep;
    float *hh = s.f(XBG_F_HH), *zb = s.f(XBG_F_ZB), *zs = s.f(XBG_F_ZS), *uu = s.f(XBG_F_UU),
          *vv = s.f(XBG_F_VV), *c = s.f(XBG_F_C), *kturb = s.f(XBG_F_KTURB),
          *rolthick = s.f(XBG_F_ROLTHICK), *dzsdt = s.f(XBG_F_DZSDT), *hu = s.f(XBG_F_HU),
          *hv = s.f(XBG_F_HV), *ueu = s.f(XBG_F_UEU), *vev = s.f(XBG_F_VEV), *H = s.f(XBG_F_H),
          *DR = s.f(XBG_F_DR), *R = s.f(XBG_F_R), *urms = s.f(XBG_F_URMS), *ceqsg = s.f(XBG_F_CEQSG),
          *cfm = s.f(XBG_F_CFM), *fwm = s.f(XBG_F_FWM), *stdep = s.f(XBG_F_STDEP), *Cc = s.f(XBG_F_CC),
          *dzb = s.f(XBG_F_DZB), *uvg = s.f(XBG_F_UV), *vug = s.f(XBG_F_VU),
          *thetamean = s.f(XBG_F_THETAMEAN);
    int *wetu = s.wetu.data(), *wetv = s.wetv.data();
    float *ceqbg = s.ceqbg.data(), *Tsg = s.Tsg.data(), *ua = s.ua.data(), *facero = s.facero.data(),
          *Sus = s.Sus.data(), *Svs = s.Svs.data(), *Sub = s.Sub.data(), *Svb = s.Svb.data(),
          *ero = s.ero.data(), *depo = s.depo.data(), *ddzb = s.ddzb.data(), *Sout = s.Sout.data();
    int *indSub = s.indSub.data(), *indSvb = s.indSvb.data();
    launch(nx, ny, [&] { longturb(nx, ny, dx, P.rho, P.g, dt, P.beta, c, kturb, rolthick, dzsdt, uu, vv, hu, hv, wetu, wetv, hh); });
    launch(nx, ny, [&] { Sbvr(nx, ny, P.rho, P.g, eps, Trep, P.D50, P.D90, P.rhosed, P.wws, P.nuhfac, ueu, vev, H, DR, R, c, hh, urms, ceqsg, ceqbg, Tsg, cfm, kturb); });
    launch(nx, ny, [&] { Rvr(nx, ny, Trep, P.facsk, P.facas, H, hh, urms, c, ua); });
    launch(nx, ny, [&] { Erosus(nx, ny, dt, P.morfac, P.por, hh, ceqsg, ceqbg, Tsg, facero, stdep); });
    launch(nx, ny, [&] { Susp(nx, ny, dx, eps, P.nuh, P.nuhfac, P.rho, P.sus, P.bed, ueu, vev, uu, uvg, hu, vv, vug, hv, zb, hh, DR, Cc, ceqbg, Sus, Svs, Sub, Svb, thetamean, ua); });
    launch(nx, ny, [&] { Conc(nx, ny, dx, dt, eps, hh, Cc, ceqsg, Tsg, facero, ero, depo, Sus, Svs); });
    launch(nx, ny, [&] { CClatbnd(nx, ny, eps, hh, Cc); });
    if (P.morfac > 0.0f) {
        launch(nx, ny, [&] { hardlayer(nx, ny, dx, dt, Sub, Svb, Sout, indSub, indSvb); });
        launch(nx, ny, [&] { zblatbnd(nx, ny, Sout); });
        launch(nx, ny, [&] { bedupdate(nx, ny, eps, dx, dt, P.morfac, P.por, hh, ero, depo, Sub, Svb, Sout, indSub, indSvb, zb, dzb, stdep); });
        launch(nx, ny, [&] { zblatbnd(nx, ny, zb); });
        launch(nx, ny, [&] { zblatbnd(nx, ny, stdep); });
        for (auto& v : s.ddzb) v = 0.0f;
        launch(nx, ny, [&] { avalanching(nx, ny, eps, dx, dt, P.por, P.drydzmax, P.wetdzmax, P.maxslpchg, hh, zb, ddzb, stdep); });
        launch(nx, ny, [&] { updatezb(nx, ny, dx, dt, zb, ddzb, dzb, zs, hh, stdep); });
        launch(nx, ny, [&] { zblatbnd(nx, ny, zb); });
        launch(nx, ny, [&] { zblatbnd(nx, ny, stdep); });
        launch(nx, ny, [&] { updatezom(nx, ny, P.cfsand, P.cfreef, P.fwsand, P.fwreef, stdep, cfm, fwm); });
    }
}
