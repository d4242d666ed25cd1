/*
 * ref_api.cpp -- TEST INFRASTRUCTURE ONLY.
 *
 * C entry points of the "reference run here" oracle (oracle/_ref).  The
 * reference's host time loop (Wave_gpu.cu) is CUDA host code and is not
 * compiled; callers pass dt, time and the boundary values of a step
 * explicitly and then run the wave / flow-boundary / flow / sediment steps.
 */
#include <cmath>
#include <cstring>
#include "ref_driver.h"

extern "C" {

int xbgr_create(const xbg_params* p, RefState** out) {
    if (!p || !out || p->nx < 4 || p->ny < 4 || p->ntheta < 1) return XBG_ERR_ARG;
    RefState* s = new RefState();
    s->P = *p;
    s->nx = p->nx; s->ny = p->ny; s->nt = p->ntheta; s->C = p->nx * p->ny;
    int C = s->C;
    for (int f = 0; f < XBG_F_COUNT; f++) {
        size_t n = C;
        if (f == XBG_F_UMEANBND) n = s->ny;
        if (f == XBG_F_EE || f == XBG_F_RR) n = (size_t)C * s->nt;
        if (f == XBG_F_WETU || f == XBG_F_WETV) n = 0;
        s->F[f].assign(n, 0.0f);
    }
    s->wetu.assign(C, 0); s->wetv.assign(C, 0);
    std::vector<float>* v2[] = {&s->sigm, &s->kh, &s->sinh2kh, &s->wci, &s->dhdx, &s->dhdy, &s->dudx,
                                &s->dudy, &s->dvdx, &s->dvdy, &s->Sxx, &s->Sxy, &s->Syy, &s->dzsdx,
                                &s->dzsdy, &s->ududx, &s->vdudy, &s->udvdx, &s->vdvdy, &s->nuh,
                                &s->viscu, &s->viscv, &s->ceqbg, &s->Tsg, &s->ua, &s->facero, &s->Sus,
                                &s->Svs, &s->Sub, &s->Svb, &s->ero, &s->depo, &s->ddzb, &s->Sout};
    for (auto* v : v2) v->assign(C, 0.0f);
    s->indSub.assign(C, 0); s->indSvb.assign(C, 0);
    size_t C3 = (size_t)C * s->nt;
    s->ctheta.assign(C3, 0.0f); s->xadv.assign(C3, 0.0f); s->yadv.assign(C3, 0.0f); s->thadv.assign(C3, 0.0f);
    s->St.assign((size_t)s->ny * s->nt, 0.0f);
    s->qbndold.assign(4 * s->ny, 0.0f); s->qbndnew.assign(4 * s->ny, 0.0f);
    s->vmeanbnd.assign(s->ny, 0.0f);
    /* theta bins (Wavestep.cu:79-86) and constants (Wave_gpu.cu:93-96) */
    s->theta.resize(s->nt); s->cxsth.resize(s->nt); s->sxnth.resize(s->nt);
    for (int i = 0; i < s->nt; i++) {
        s->theta[i] = (float)(i * (p->dtheta) + p->thetamin + 0.5f * p->dtheta);
        s->cxsth[i] = cosf(s->theta[i]);
        s->sxnth[i] = sinf(s->theta[i]);
    }
    float phi = (1.0f + sqrtf(5.0f)) / 2;
    s->aphi = 1 / (phi + 1);
    s->bphi = phi / (phi + 1);
    s->twopi = 8 * atanf(1.0f);
    *out = s;
    return XBG_OK;
}
int xbgr_destroy(RefState* s) { delete s; return XBG_OK; }

int xbgr_set_field(RefState* s, int id, const void* p, size_t n) {
    if (id < 0 || id >= XBG_F_COUNT) return XBG_ERR_ARG;
    if (id == XBG_F_WETU || id == XBG_F_WETV) {
        if (n != (size_t)s->C) return XBG_ERR_ARG;
        std::memcpy(id == XBG_F_WETU ? s->wetu.data() : s->wetv.data(), p, n * sizeof(int));
        return XBG_OK;
    }
    if (n != s->F[id].size()) return XBG_ERR_ARG;
    std::memcpy(s->F[id].data(), p, n * sizeof(float));
    return XBG_OK;
}
int xbgr_get_field(RefState* s, int id, void* p, size_t n) {
    if (id < 0 || id >= XBG_F_COUNT) return XBG_ERR_ARG;
    if (id == XBG_F_WETU || id == XBG_F_WETV) {
        if (n != (size_t)s->C) return XBG_ERR_ARG;
        std::memcpy(p, id == XBG_F_WETU ? s->wetu.data() : s->wetv.data(), n * sizeof(int));
        return XBG_OK;
    }
    if (n != s->F[id].size()) return XBG_ERR_ARG;
    std::memcpy(p, s->F[id].data(), n * sizeof(float));
    return XBG_OK;
}
/* The per-step inputs that the reference host code computes:
 * dt, totaltime (Wave_gpu.cu:696-698), Trep and St (wavebnd), qbndold/new,
 * timesincelast/timenext, zsbndi/zsbndn, windu/windv (flowbnd).            */
int xbgr_set_step_inputs(RefState* s, double dt, double totaltime, float Trep, const float* St,
                         const float* qold, const float* qnew, float timesincelast, float timenext,
                         float zsbndi, float zsbndn, float windu, float windv) {
    s->dt = dt; s->totaltime = totaltime; s->Trep = Trep;
    if (St) std::memcpy(s->St.data(), St, s->St.size() * sizeof(float));
    if (qold) std::memcpy(s->qbndold.data(), qold, s->qbndold.size() * sizeof(float));
    if (qnew) std::memcpy(s->qbndnew.data(), qnew, s->qbndnew.size() * sizeof(float));
    s->timesincelast = timesincelast; s->timenext = timenext;
    s->zsbndi = zsbndi; s->zsbndn = zsbndn; s->windu = windu; s->windv = windv;
    return XBG_OK;
}
int xbgr_wave_step(RefState* s) { ref_wave_step_cpu(*s); return XBG_OK; }
int xbgr_flow_boundary(RefState* s) { ref_flow_boundary(*s); return XBG_OK; }
int xbgr_flow_step(RefState* s) { ref_flow_step(*s); return XBG_OK; }
int xbgr_sediment_step(RefState* s) { ref_sediment_step(*s); return XBG_OK; }

}  // extern "C"
