/*
 * xbg_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of the reference's coupled step, used by tests/, by
 * __graft_entry__.smoke() and by bench.py's CPU-baseline leg as the checker.
 * Nothing in the product links or calls it.  The API mirrors include/xbg.h
 * one for one (xbgo_* <-> xbg_*), so a parity test drives both the same way.
 *
 * Semantics: kernel-by-kernel in the reference's launch order, every kernel
 * reading a snapshot of its inputs (Jacobi) where the reference GPU code
 * races; the documented deviations are listed in xbg_oracle.cpp's header.
 */
#ifndef XBG_ORACLE_H
#define XBG_ORACLE_H
#include "../include/xbg.h"
#ifdef __cplusplus
extern "C" {
#endif
typedef struct xbgo xbgo;
int  xbgo_create(const xbg_params* p, int precision, xbgo** out);
int  xbgo_destroy(xbgo* o);
int  xbgo_init_state(xbgo* o, const void* zb, double zs0, double zs1);
int  xbgo_field_count(const xbgo* o, int field, size_t* count);
int  xbgo_set_field(xbgo* o, int field, const void* host, size_t count);
int  xbgo_get_field(xbgo* o, int field, void* host, size_t count);
int  xbgo_set_wave_boundary(xbgo* o, int slot, const double* St,
                            const double* qbnd, int nrec, const double* times,
                            double t0, double tend, double Trep);
int  xbgo_set_sealevel(xbgo* o, const double* time, const double* w0,
                       const double* w1, int n);
int  xbgo_set_wind(xbgo* o, const double* time, const double* U,
                   const double* V, int n);
int  xbgo_compute_dt(xbgo* o);
int  xbgo_wave_boundary(xbgo* o);
int  xbgo_flow_boundary(xbgo* o);
int  xbgo_wave_step(xbgo* o);
int  xbgo_flow_step(xbgo* o);
int  xbgo_sediment_step(xbgo* o);
int  xbgo_accumulate_means(xbgo* o);
int  xbgo_step(xbgo* o);
int  xbgo_advance(xbgo* o, int nsteps);
int  xbgo_get_time(xbgo* o, double* totaltime, double* dt, int64_t* nstep,
                   int* flags);
int  xbgo_set_time(xbgo* o, double totaltime, double dt, double wdt);
int  xbgo_output_done(xbgo* o);
int  xbgo_reset_means(xbgo* o);
int  xbgo_mass(xbgo* o, double* water, double* sed, double* bed);
#ifdef __cplusplus
}
#endif
#endif
