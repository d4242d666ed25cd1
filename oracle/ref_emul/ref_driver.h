/*
 * ref_driver.h -- TEST INFRASTRUCTURE ONLY.
 *
 * State of the "reference run here" oracle: the reference's own wave_CPU.cpp
 * functions and its own CUDA kernel sources (run on the CPU through
 * cuda_emul.h), driven in the launch order of the reference host functions.
 * FP32 only, like the reference (DECNUM = float, XBeachGPU.h:37).
 */
#ifndef XBG_REF_DRIVER_H
#define XBG_REF_DRIVER_H
#include <vector>
#include "../../include/xbg.h"

struct RefState {
    xbg_params P;
    int nx, ny, nt, C;
    std::vector<float> F[XBG_F_COUNT];
    std::vector<int> wetu, wetv;
    std::vector<float> theta, cxsth, sxnth;
    /* step inputs set explicitly by the caller (host logic is not compiled) */
    double dt = 0, totaltime = 0;
    float Trep = 10, timesincelast = 0, timenext = 1, zsbndi = 0, zsbndn = 0;
    float windu = 0, windv = 0;
    std::vector<float> St, qbndold, qbndnew, vmeanbnd;
    /* temporaries of wavestep / flowstep / sedimentstep */
    std::vector<float> sigm, kh, sinh2kh, wci, ctheta, xadv, yadv, thadv,
        dhdx, dhdy, dudx, dudy, dvdx, dvdy, Sxx, Sxy, Syy, dzsdx, dzsdy,
        ududx, vdudy, udvdx, vdvdy, nuh, viscu, viscv, ceqbg, Tsg, ua, facero,
        Sus, Svs, Sub, Svb, ero, depo, ddzb, Sout;
    std::vector<int> indSub, indSvb;
    float twopi, aphi, bphi;
    float* f(int id) { return F[id].data(); }
};

void ref_wave_step_cpu(RefState& s);          /* ref_wave.cpp    */
void ref_flow_boundary(RefState& s);            /* ref_kernels.cpp */
void ref_flow_step(RefState& s);
void ref_sediment_step(RefState& s);
#endif
