// Stand-ins for the reference's host types that the binding in
// xbg_binding.cpp reads: XBGPUParam (XBeachGPU.h:62-154), SLBnd
// (XBeachGPU.h:176), WindBnd (:182) and Wavebndparam (:198).  Same member
// names and meaning, only the members the binding uses.  A reference build
// includes XBeachGPU.h instead of this file; the test driver uses it so the
// binding compiles and runs without the reference's sources.
#ifndef XBG_TEST_REF_HOST_TYPES_H
#define XBG_TEST_REF_HOST_TYPES_H
#include <string>
#include <vector>

struct XBGPUParam {
    int nx = 0, ny = 0;
    double dx = 0.0;
    int swave = 1, flow = 1, sedtrans = 0, morphology = 0;
    double g = 9.81, rho = 1025.0, eps = 0.01;
    double cf = 0.01, cfsand = 0.0, cfreef = 0.0;
    double nuh = 1.0, nuhfac = 1.0;
    int usesmago = 1;
    double smag = 0.3, lat = 0.0, fc = 0.0, Cd = 0.002;
    double wci = 0.0, hwci = 0.1;
    int breakmodel = 1;
    double gammaa = 0.6, n = 8.0, alpha = 1.0, gammax = 2.0, beta = 0.15;
    double fw = 0.001, fwsand = 0.0, fwreef = 0.0;
    int roller = 1;
    double thetamin = -90.0 * 3.14159265 / 180.0, thetamax = 90.0 * 3.14159265 / 180.0, dtheta = 0.0;
    double D50 = 0.00038, D90 = 0.00053, rhosed = 2650.0, wws = 0.0509;
    double drydzmax = 1.0, wetdzmax = 0.3, maxslpchg = 0.01, por = 0.4, morfac = 1.0;
    double sus = 1.0, bed = 1.0, facsk = 0.2, facas = 0.2;
    int wavebndtype = 2;
    double CFL = 0.7, sedstart = 3600.0, outputtimestep = 0.0, endtime = 0.0;
    double dtbc = 1.0, rtlength = 3600.0;
    std::string outfile = "XBGPU_output.nc";
    std::vector<std::string> outvars;
};

struct SLBnd { double time, wlev0, wlev1; };
struct WindBnd { double time, U, V, spd, dir, theta; };
struct Wavebndparam { double time, Hs, Tp, Dp, s, gamma = 3.3, alpha = 1.0, Trep = 0.0; };

#endif
