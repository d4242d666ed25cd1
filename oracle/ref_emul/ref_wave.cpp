/*
 * ref_wave.cpp -- TEST INFRASTRUCTURE ONLY.
 *
 * Calls the reference's own CPU wave functions (wave_CPU.cpp, compiled in
 * place from the reference checkout) in the order of wavestepCPU,
 * Wavestep.cu:1169-1302.  The reference's header is used for the
 * prototypes; netcdf.h / fftw3.h resolve to the stubs in oracle/stubs.
 */
#include "XBeachGPU.h"
#include "ref_driver.h"

void ref_wave_step_cpu(RefState& s) {
    int nx = s.nx, ny = s.ny, ntheta = s.nt;
    DECNUM dtheta = (DECNUM)s.P.dtheta;
    DECNUM* ee = s.f(XBG_F_EE); DECNUM* rr = s.f(XBG_F_RR);
    DECNUM* hh = s.f(XBG_F_HH); DECNUM* uu = s.f(XBG_F_UU); DECNUM* vv = s.f(XBG_F_VV);
    DECNUM* k = s.f(XBG_F_K); DECNUM* c = s.f(XBG_F_C); DECNUM* cg = s.f(XBG_F_CG);
    DECNUM* E = s.f(XBG_F_E); DECNUM* H = s.f(XBG_F_H); DECNUM* D = s.f(XBG_F_D);
    DECNUM* DR = s.f(XBG_F_DR); DECNUM* R = s.f(XBG_F_R);
    DECNUM* fwm = s.f(XBG_F_FWM); DECNUM* cfm = s.f(XBG_F_CFM);
    DECNUM* thetamean = s.f(XBG_F_THETAMEAN);
    DECNUM* Fx = s.f(XBG_F_FX); DECNUM* Fy = s.f(XBG_F_FY);
    DECNUM* urms = s.f(XBG_F_URMS); DECNUM* ust = s.f(XBG_F_UST);
    DECNUM* sigm = s.sigm.data(); DECNUM* kh = s.kh.data(); DECNUM* sinh2kh = s.sinh2kh.data();
    DECNUM* wci = s.wci.data(); DECNUM* ctheta = s.ctheta.data();
    DECNUM* dhdx = s.dhdx.data(); DECNUM* dhdy = s.dhdy.data(); DECNUM* dudx = s.dudx.data();
    DECNUM* dudy = s.dudy.data(); DECNUM* dvdx = s.dvdx.data(); DECNUM* dvdy = s.dvdy.data();
    DECNUM* xadvec = s.xadv.data(); DECNUM* yadvec = s.yadv.data(); DECNUM* thetaadvec = s.thadv.data();
    DECNUM* cxsth = s.cxsth.data(); DECNUM* sxnth = s.sxnth.data(); DECNUM* theta = s.theta.data();
    DECNUM* Sxx = s.Sxx.data(); DECNUM* Sxy = s.Sxy.data(); DECNUM* Syy = s.Syy.data();
    DECNUM* St = s.St.data();
    XBGPUParam Param;
    Param.dt = s.dt; Param.dx = s.P.dx; Param.eps = s.P.eps; Param.g = s.P.g; Param.rho = s.P.rho;
    Param.wci = s.P.wci; Param.hwci = s.P.hwci; Param.gammax = s.P.gammax; Param.gammaa = s.P.gammaa;
    Param.alpha = s.P.alpha; Param.n = s.P.n; Param.beta = s.P.beta; Param.breakmodel = s.P.breakmodel;
    DECNUM Trep = s.Trep;
    double totaltime = s.totaltime;

    offshorebndWavCPU(nx, ny, ntheta, totaltime, Trep, St, sigm, ee);
    sanityCPU(nx, ny, Param.eps, hh, sigm, ntheta, ee);
    dispersionCPU(nx, ny, s.twopi, Param.g, s.aphi, s.bphi, sigm, hh, k, c, kh, sinh2kh, cg);
    calcwciCPU(nx, ny, Param.wci, Param.hwci, hh, wci);
    slopesCPU(nx, ny, Param.dx, hh, uu, vv, dhdx, dhdy, dudx, dudy, dvdx, dvdy);
    propagthetaCPU(nx, ny, ntheta, wci, ctheta, cxsth, sxnth, dhdx, dhdy, dudx, dudy, dvdx, dvdy, sigm, kh);
    actionCPU(ntheta, nx, ny, ee, sigm);
    xadvecupwind2CPU(nx, ny, ntheta, dtheta, Param.dx, Param.dt, wci, ee, cg, cxsth, uu, xadvec);
    yadvecupwind2CPU(nx, ny, ntheta, dtheta, Param.dx, Param.dt, wci, ee, cg, sxnth, vv, yadvec);
    thetaadvecuw2hoCPU(nx, ny, ntheta, dtheta, Param.dx, Param.dt, Param.wci, ee, ctheta, thetaadvec);
    eulerupwindCPU(nx, ny, ntheta, dtheta, Param.dx, Param.dt, Param.wci, ee, xadvec, yadvec, thetaadvec);
    rollerlatbndCPU(nx, ny, ntheta, Param.eps, hh, ee);
    energyCPU(nx, ny, ntheta, ee, sigm);
    energintCPU(nx, ny, ntheta, dtheta, Param.rho, Param.g, Param.gammax, E, H, hh, ee);
    if (Param.breakmodel == 1)
        roelvinkCPU(nx, ny, Param.rho, Param.g, Param.gammaa, Param.alpha, Param.n, Trep, fwm, cfm, hh, H, E, D, k);
    else
        baldockCPU(nx, ny, Param.rho, Param.g, Param.gammaa, Param.alpha, Param.n, Trep, fwm, cfm, hh, H, E, D, k);
    if (s.P.roller == 1) {
        xadvecupwind2CPU(nx, ny, ntheta, dtheta, Param.dx, Param.dt, wci, rr, c, cxsth, uu, xadvec);
        yadvecupwind2CPU(nx, ny, ntheta, dtheta, Param.dx, Param.dt, wci, rr, c, sxnth, vv, yadvec);
        thetaadvecuw2hoCPU(nx, ny, ntheta, dtheta, Param.dx, Param.dt, Param.wci, rr, ctheta, thetaadvec);
        eulerupwindCPU(nx, ny, ntheta, dtheta, Param.dx, Param.dt, Param.wci, rr, xadvec, yadvec, thetaadvec);
        rollerlatbndCPU(nx, ny, ntheta, Param.eps, hh, rr);
    }
    dissipationCPU(nx, ny, ntheta, dtheta, Param.eps, Param.dt, Param.g, Param.beta, wci, hh, ee, D, E, rr, c, cxsth, sxnth, uu, vv, DR, R);
    rollerlatbndCPU(nx, ny, ntheta, Param.eps, hh, ee);
    meandirCPU(nx, ny, ntheta, Param.rho, Param.g, dtheta, ee, theta, thetamean, E, H);
    radstressCPU(nx, ny, ntheta, Param.dx, dtheta, ee, rr, cxsth, sxnth, cg, c, Sxx, Sxy, Syy);
    wavforceCPU(nx, ny, ntheta, Param.dx, dtheta, Sxx, Sxy, Syy, Fx, Fy, hh);
    twodimbndnoixCPU(nx, ny, Param.eps, hh, Fx);
    twodimbndCPU(nx, ny, Param.eps, hh, Fy);
    breakerdelayCPU(nx, ny, ntheta, dtheta, Param.g, Param.rho, Trep, Param.eps, urms, ust, H, E, c, k, hh, R);
    twodimbndCPU(nx, ny, Param.eps, hh, ust);
}
