/*
 * xbg.h -- C ABI of the B200-native XBeach_GPU coupled step.
 *
 * This header is the drop-in boundary for the reference's per-timestep path:
 * the host step functions declared in XBeachGPU.h:348-353
 *     void wavebnd(XBGPUParam, std::vector<Wavebndparam>);        (Wavestep.cu:512)
 *     void flowbnd(XBGPUParam, slbnd, wndbnd, wavebnd);           (Wave_gpu.cu:1020)
 *     void wavestep(XBGPUParam);                                   (Wavestep.cu:755)
 *     void flowstep(XBGPUParam);                                   (Wave_gpu.cu:1106)
 *     void sedimentstep(XBGPUParam);                               (Wave_gpu.cu:1405)
 * plus the dt logic and running means of one mainloopGPU iteration
 * (Wave_gpu.cu:610-757).  The reference keeps its state in ~120 file-scope
 * device pointers (Wave_gpu.cu:26-241); here the state lives behind an opaque
 * handle that owns all device memory.  Plain C types only: pointers, sizes,
 * ints and doubles.
 *
 * Conventions
 *  - Every call returns an int status (XBG_OK or an XBG_ERR_* code); no call
 *    exits the process (the reference calls exit() from CUDA_CHECK,
 *    Wavestep.cu:4-18, and on a NaN dt, Wave_gpu.cu:642-647).
 *  - Grid layout is the reference's: structure of arrays, cell i = ix + iy*nx
 *    (x cross-shore, offshore boundary at ix = 0), directional fields stored as
 *    theta-planes f[i + itheta*nx*ny] (Wave_kernel.cu:264).
 *  - zb is bed depth, positive down; hh = zb + zs (Wave_gpu.cu:2009-2010).
 *  - Field values are float for an XBG_FP32 handle and double for an XBG_FP64
 *    handle, except the wet flags (int32).  Time and dt are always double.
 *  - All device work of a handle is ordered on one handle-owned CUDA stream.
 *    Calls that return host data synchronise that stream; the others do not.
 *    One handle must not be used from two host threads at once.
 */
#ifndef XBG_H
#define XBG_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define XBG_OK            0
#define XBG_ERR_ARG       1  /* bad argument or size                          */
#define XBG_ERR_CUDA      2  /* a CUDA runtime call failed                    */
#define XBG_ERR_NAN       3  /* dt became 0, inf or NaN: "Model crashed!"     */
#define XBG_ERR_DT        4  /* initial dt below 1e-8 (Wave_gpu.cu:2670-2677) */
#define XBG_ERR_TIMEOUT   5  /* a bounded device wait ran out                 */
#define XBG_ERR_STATE     6  /* call out of order (e.g. no wave boundary set) */
#define XBG_ERR_NOMEM     7  /* device allocation failed                      */
#define XBG_ERR_BOUNDARY  8  /* time ran past the last uploaded boundary data */
#define XBG_ERR_IO        9  /* a file could not be opened or written        */
#define XBG_ERR_FORMAT   10  /* an input file does not have the expected form */

#define XBG_FP32 0
#define XBG_FP64 1

/* ---- parameters (XBGPUParam, XBeachGPU.h:62-154) ------------------------
 * Angles are in radians (the parameter file gives degrees and read_input.cpp
 * converts them).  xbg_params_default() fills the reference defaults;
 * xbg_params_sanity() applies the cross-parameter rules of checkparamsanity
 * (read_input.cpp:1227-1443) that bear on the step path.                    */
typedef struct xbg_params {
    int    nx, ny;          /* grid size                                    */
    double dx;              /* grid spacing [m]                             */
    int    swave, flow, sedtrans, morphology;
    double g, rho, eps;     /* gravity, water density, drying height        */
    double cf, cfsand, cfreef;       /* bottom friction                     */
    double nuh, nuhfac;     /* viscosity (nuh = smag when usesmago = 1)     */
    int    usesmago;
    double smag;
    double lat, fc, Cd;     /* latitude [rad], Coriolis, wind drag          */
    double wci, hwci;       /* wave-current interaction switch, min depth   */
    int    breakmodel;      /* 1 Roelvink, 2 Baldock                        */
    double gammaa, n, alpha, gammax, beta;
    double fw, fwsand, fwreef;
    int    roller;          /* roller model on/off                          */
    double thetamin, thetamax, dtheta;   /* directional bins [rad]          */
    int    ntheta;
    double D50, D90, rhosed, wws, drydzmax, wetdzmax, maxslpchg, por,
           morfac, sus, bed, facsk, facas;
    int    wavebndtype;     /* 1 constant records, >=2 wave-group chunks    */
    double CFL, sedstart, outputtimestep, endtime;
    double dtbc, rtlength;  /* wave-group record step and chunk length [s]  */
    int    means;           /* accumulate running means every step (1)      */
} xbg_params;

void xbg_params_default(xbg_params* p);
/* endbnd: time of the last boundary record (min over sea level, wind and
 * wave series), used to clamp endtime as checkparamsanity does.           */
int  xbg_params_sanity(xbg_params* p, double endbnd);

/* ---- fields ------------------------------------------------------------- */
enum xbg_field {
    XBG_F_ZB = 0, XBG_F_ZS, XBG_F_HH, XBG_F_UU, XBG_F_VV,
    XBG_F_HU, XBG_F_HV, XBG_F_HUM, XBG_F_HVM, XBG_F_QX, XBG_F_QY,
    XBG_F_UEU, XBG_F_VEV, XBG_F_VMAGEU, XBG_F_VMAGEV, XBG_F_VU, XBG_F_UV,
    XBG_F_UUOLD, XBG_F_VVOLD, XBG_F_ZSOLD, XBG_F_DZSDT,
    XBG_F_H, XBG_F_E, XBG_F_D, XBG_F_DR, XBG_F_R,
    XBG_F_K, XBG_F_C, XBG_F_CG, XBG_F_FX, XBG_F_FY, XBG_F_URMS, XBG_F_UST,
    XBG_F_THETAMEAN, XBG_F_CFM, XBG_F_FWM,
    XBG_F_CC, XBG_F_CEQSG, XBG_F_STDEP, XBG_F_DZB, XBG_F_ROLTHICK, XBG_F_KTURB,
    XBG_F_HMEAN, XBG_F_UUMEAN, XBG_F_VVMEAN, XBG_F_HHMEAN, XBG_F_ZSMEAN,
    XBG_F_CMEAN, XBG_F_ZSMAX,
    XBG_F_WETU, XBG_F_WETV,          /* int32 flags                        */
    XBG_F_UMEANBND,                  /* ny values (ubnd1D running mean)    */
    XBG_F_EE, XBG_F_RR,              /* nx*ny*ntheta (theta-planes)        */
    XBG_F_COUNT
};

/* ---- lifecycle ---------------------------------------------------------- */
typedef struct xbg_handle xbg_handle;

/* Allocates all device state for p (after xbg_params_sanity) on the current
 * CUDA device and sets the reference's initial condition for the constant
 * parts (theta bins Wavestep.cu:79-86; Wave_gpu.cu:1988-2015, 2187-2510).
 * Fields are zero until set with xbg_set_field / xbg_init_state.          */
int  xbg_create(const xbg_params* p, int precision, xbg_handle** out);
int  xbg_destroy(xbg_handle* h);
const char* xbg_status_string(int status);

/* Reference initial state from bathymetry zb and the first sea-level record
 * (Wave_gpu.cu:1988-2015, 2519-2551, 2637-2692): zs, hh, hu/hv/hum/hvm = hh,
 * stdep = 5 m, cfm/fwm by updatezom, initial dt = 0.5*min(0.5*CFL*dx/sqrt(g h)),
 * ee column 0 from the first boundary record.  zb: nx*ny host values.      */
int  xbg_init_state(xbg_handle* h, const void* zb, double zs0, double zs1);

/* ---- state IO ----------------------------------------------------------- */
int  xbg_field_count(const xbg_handle* h, int field, size_t* count);
int  xbg_set_field(xbg_handle* h, int field, const void* host, size_t count);
int  xbg_get_field(xbg_handle* h, int field, void* host, size_t count);
/* Zero-copy access: the device pointer of a field (owned by the handle). */
int  xbg_field_device_ptr(xbg_handle* h, int field, void** dptr, size_t* count);
/* ee (wave energy per bin) is non-negative in memory: xbg_set_field clips
 * negative values to 0 (the reference's sanity step, Wave_kernel.cu:324,
 * applied when the state is set); values written through the device
 * pointer must be >= 0.                                                     */

/* ---- boundaries ----------------------------------------------------------
 * Wave boundary data of one chunk: St[nrec][ntheta][ny] (Stfile layout
 * Wavestep.cu:703-706) and qbnd[nrec][4][ny] (qfile layout :709-712), with
 * record times t0 + m*dtbc (wavebndtype >= 2) or times[m] (wavebndtype 1).
 * Trep: representative period of the chunk.  The per-step interpolation of
 * wavebnd (Wavestep.cu:684-741) runs on the device.  A second chunk may be
 * queued while the first is in use (slot = 0 current, 1 next).            */
int  xbg_set_wave_boundary(xbg_handle* h, int slot, const double* St,
                           const double* qbnd, int nrec, const double* times,
                           double t0, double tend, double Trep);
/* Overwrite records [first, first+n) of a queued or current chunk from host
 * memory in the handle's element type (float for XBG_FP32), stream-ordered
 * and without synchronising: boundary records streamed while the model runs.
 * St: n*ntheta*ny values, q: n*4*ny values.                                */
int  xbg_put_wave_records(xbg_handle* h, int slot, int first, int n,
                          const void* St, const void* q);
/* Sea-level records (time, wlev0, wlev1) and wind records (time, U, V),
 * interpolated on the device each step as flowbnd does
 * (Wave_gpu.cu:1020-1103).                                                 */
int  xbg_set_sealevel(xbg_handle* h, const double* time, const double* wlev0,
                      const double* wlev1, int n);
int  xbg_set_wind(xbg_handle* h, const double* time, const double* U,
                  const double* V, int n);

/* ---- stepping ----------------------------------------------------------
 * The pieces of one mainloopGPU iteration, in the reference's order.  Each
 * enqueues device work only; dt and time live on the device.             */
int  xbg_compute_dt(xbg_handle* h);        /* Wave_gpu.cu:620-698          */
int  xbg_wave_boundary(xbg_handle* h);     /* wavebnd, Wavestep.cu:512     */
int  xbg_flow_boundary(xbg_handle* h);     /* flowbnd, Wave_gpu.cu:1020    */
int  xbg_wave_step(xbg_handle* h);         /* wavestep, Wavestep.cu:755    */
int  xbg_flow_step(xbg_handle* h);         /* flowstep, Wave_gpu.cu:1106   */
int  xbg_sediment_step(xbg_handle* h);     /* sedimentstep, :1405 (runs only
                                              when sedtrans=1, t>=sedstart) */
int  xbg_accumulate_means(xbg_handle* h);  /* Wave_gpu.cu:731-757          */
/* One whole coupled step (all of the above), replayed from a CUDA graph. */
int  xbg_step(xbg_handle* h);
/* Up to nsteps coupled steps; steps after the device reaches endtime, an
 * output time or an error are skipped on the device.  Does not synchronise. */
int  xbg_advance(xbg_handle* h, int nsteps);
/* Synchronise and read time, dt, step count and the device status word.  */
int  xbg_get_time(xbg_handle* h, double* totaltime, double* dt, int64_t* nstep,
                  int* flags);
/* The same without waiting: copies the device clock (XBG_CLOCK_BYTES
 * bytes) into dst (pinned host memory) in the handle's stream order; once
 * the stream has passed the copy, xbg_clock_decode reads it (and returns
 * the status word) as xbg_get_time would have at that point of the stream. */
#define XBG_CLOCK_BYTES 240
/* Checkpoint / resume (the reference has none: its hot start is commented
 * out, Wave_gpu.cu:2973-2984).  One host buffer holds every buffer that
 * carries state from step to step -- the persistent fields, both plane sets
 * of ee and rr, the previous level, the running means, the WAVEDT partials,
 * the boundary slots and series, and the device clock (time, dt, step
 * counters, boundary cursors, status) -- behind a header naming the grid and
 * precision.  Loading it into a handle created with the same parameters
 * continues the run bit for bit; a buffer of another grid or precision is
 * XBG_ERR_ARG.  A scenario of a batch takes only a snapshot whose boundary
 * slots have its own capacity (else XBG_ERR_STATE).  Both synchronise the
 * handle's stream.                                                        */
int  xbg_state_bytes(xbg_handle* h, size_t* bytes);
int  xbg_save_state(xbg_handle* h, void* dst, size_t bytes);
int  xbg_load_state(xbg_handle* h, const void* src, size_t bytes);
int  xbg_get_time_async(xbg_handle* h, void* dst);
int  xbg_clock_decode(xbg_handle* h, const void* src, double* totaltime, double* dt,
                      int64_t* nstep, int* flags);
#define XBG_FLAG_OUTPUT_DUE   1   /* nextoutputtime reached               */
#define XBG_FLAG_ENDED        2   /* totaltime >= endtime                 */
#define XBG_FLAG_NEED_BOUNDARY 4  /* next wave-boundary chunk consumed    */
#define XBG_FLAG_FALLBACK     8   /* batch scenario left surrogate forcing
                                     for the plain wave solver for good    */
/* Output bookkeeping of mainloopGPU (Wave_gpu.cu:784-930): divide the means
 * by the step count, advance nextoutputtime; xbg_reset_means clears them. */
int  xbg_output_done(xbg_handle* h);
int  xbg_reset_means(xbg_handle* h);
/* Set time and dt directly (e.g. to replay a fixed-dt sequence). */
int  xbg_set_time(xbg_handle* h, double totaltime, double dt, double wdt);
int  xbg_sync(xbg_handle* h);

/* ---- diagnostics -------------------------------------------------------- */
/* Number of kernel launches this handle has enqueued since creation. */
int  xbg_launch_count(const xbg_handle* h, int64_t* count);
/* The handle's CUDA stream (a cudaStream_t), for callers that time or order
 * their own work against the model's. */
int  xbg_get_stream(xbg_handle* h, void** stream);
/* Run one coupled step without the graph, with a CUDA event after every
 * kernel; returns each kernel's duration [ms] and name.  *n: in = capacity,
 * out = kernels run.                                                      */
int  xbg_profile_step(xbg_handle* h, float* ms, const char** names, int* n);
/* Kernel variants of a phase, for comparison and tuning.  Phase
 * XBG_PHASE_WAVE (the fused wave rows pass): variants 1 and 2 move its plane
 * tiles with the tensor memory accelerator (box copies issued by one thread
 * per block; available when wave-current interaction is off and nx is a
 * multiple of 4) with one or two cells per thread, variant 0 copies them
 * with every thread (cp.async).  Phase XBG_PHASE_FLOW: variant 1 runs
 * eulerustep and eulervstep as one pass (uu* of the block's tile and its
 * ring in shared memory), variant 0 as two.  All variants of a phase give
 * the same results bit for bit.  Setting a variant that does not apply is
 * XBG_ERR_ARG; get reports the one in use.  Phase XBG_PHASE_TILE: the tile
 * shape of the passes that read only a cell and its nearest neighbours
 * (wavforce, the depth/viscosity and momentum passes, the first sediment
 * pass): variant 0 blocks of 32 x 8 cells, variant 1 blocks of 64 x 4;
 * variant 2 (single domain, nx a multiple of 4 in FP32 or 2 in FP64; the
 * default there) runs the depth/viscosity pass and the first sediment pass
 * over row segments, 4 (2) cells per thread with 16-byte loads, and the
 * others in 32 x 8 blocks.                                                 */
#define XBG_PHASE_WAVE 0
#define XBG_PHASE_FLOW 1
#define XBG_PHASE_TILE 2
int  xbg_set_kernel_variant(xbg_handle* h, int phase, int variant);
int  xbg_get_kernel_variant(xbg_handle* h, int phase, int* variant);
/* Device-side water and sediment ledgers (sum zs*dx^2, sum (C*h) dx^2,
 * sum zb dx^2) in double, computed on the device.                         */
int  xbg_mass(xbg_handle* h, double* water, double* sediment_susp,
              double* bed);

/* ---- wave forcing from outside the wave solver ---------------------------
 * No counterpart in the reference.  Sets the wave forcing fields E, H, D,
 * DR, Fx, Fy to f0 + w (f1 - f0) (E, H, D, DR clipped at 0), where f0 and f1
 * are host arrays of six DEVICE plane pointers of the handle's precision
 * (the surrogate's predictions); with rescale != 0 the wave action of every
 * bin and the roller energy are scaled per cell to the new E and DR, so a
 * later plain wave step continues from the state the forcing describes.
 * Enqueued on the handle's stream; used between xbg_flow_boundary and
 * xbg_flow_step in place of xbg_wave_step.                                   */
int  xbg_set_wave_forcing(xbg_handle* h, const void* const* f0,
                          const void* const* f1, double w, int rescale);
/* No counterpart in the reference.  k coupled steps in which the forcing
 * replaces the wave sub-step: step j = 1..k runs the dt pass, ubnd1D,
 * xbg_set_wave_forcing(f0, f1, j/k, rescale = (j == k)), flow, sediment and
 * means -- the same kernels in the same order as those calls made one by one
 * -- replayed from one CUDA graph captured on the first call for this
 * (f0, f1, k).  Enqueued on the handle's stream; the planes must stay valid
 * while it runs.                                                             */
int  xbg_forcing_steps(xbg_handle* h, const void* const* f0,
                       const void* const* f1, int k);

/* ---- batches of scenarios ------------------------------------------------
 * No counterpart in the reference (it runs one grid per process).  A batch
 * advances n scenarios -- each its own grid size, parameters, boundaries,
 * clock and dt -- with one launch per kernel of the step for all of them,
 * replayed from one CUDA graph.  The scenarios share precision, ntheta and
 * the swave/flow/sedtrans/roller/means switches (XBG_ERR_ARG otherwise).
 * Each scenario is an ordinary handle owned by the batch: set fields,
 * boundaries and time, and read results, with the xbg_* calls above on the
 * handle from xbg_batch_scenario (reads wait for the batch's stream);
 * stepping a scenario's handle on its own is not supported while it is in
 * a batch, and xbg_destroy refuses it (XBG_ERR_STATE).                    */
typedef struct xbg_batch xbg_batch;
#define XBG_MAX_BATCH 4096
int  xbg_batch_create(const xbg_params* params, int n, int precision,
                      xbg_batch** out);            /* params: n entries   */
int  xbg_batch_destroy(xbg_batch* b);
int  xbg_batch_scenario(xbg_batch* b, int s, xbg_handle** h);
/* nsteps coupled steps of every scenario (each with its own dt; a scenario
 * that reached its end time, an output time or an error skips them).  Does
 * not synchronise.                                                          */
int  xbg_batch_advance(xbg_batch* b, int nsteps);
/* Synchronise and read every scenario's time, dt, steps, flags and status
 * word (arrays of n; any may be NULL).                                      */
int  xbg_batch_status(xbg_batch* b, double* t, double* dt, int64_t* nstep,
                      int* flags, int* status);
int  xbg_batch_sync(xbg_batch* b);
int  xbg_batch_get_stream(xbg_batch* b, void** stream);
/* As xbg_profile_step, for one batched step. */
int  xbg_batch_profile_step(xbg_batch* b, float* ms, const char** names,
                            int* n);
/* Persistent blocks of the launches of one tile shape (0: 32x8 tiles,
 * 1: wave rows, 2: 256-cell runs, 3: one block per scenario, 4: boundary
 * values, 5: dt reduction, 6: 64x4 tiles); used by the autotuner. */
int  xbg_batch_set_grid(xbg_batch* b, int shape, int blocks);
int  xbg_batch_launch_count(xbg_batch* b, int64_t* count);
/* As xbg_set_kernel_variant, for every scenario of a batch (the TMA rows
 * pass needs every scenario eligible).  Used by the autotuner.             */
int  xbg_batch_set_kernel_variant(xbg_batch* b, int phase, int variant);
int  xbg_batch_get_kernel_variant(xbg_batch* b, int phase, int* variant);

/* ---- surrogate-assisted batches --------------------------------------
 * No counterpart in the reference (its wave sub-stepping, nwstp of
 * Wave_gpu.cu:77 and wavebndOLD of Wavestep.cu:386, was removed).  Each
 * scenario's wave sub-step is either the plain wave solver or a forcing
 * given from outside (the surrogate's predictions), per scenario:       */
#define XBG_WAVE_PLAIN    0   /* the wave solver runs                      */
#define XBG_WAVE_FORCED   1   /* E, H, D, DR, Fx, Fy come from the forcing */
#define XBG_WAVE_FALLBACK 2   /* plain, and XBG_FLAG_FALLBACK is set (the
                                 scenario failed its judge)                */
/* Stream-ordered on the batch's stream.  FORCED needs forcing planes.      */
int  xbg_batch_set_wave_mode(xbg_batch* b, int s, int mode);
/* Scenario s's forcing: six device planes each of f0 (the fields at the
 * segment start) and f1 (the fields predicted at its end), in the order
 * E, H, D, DR, Fx, Fy, element type of the batch, nx*ny values each.     */
int  xbg_batch_set_forcing(xbg_batch* b, int s, const void* const* f0,
                           const void* const* f1);
/* k coupled steps of every scenario (one CUDA graph per k, replayed): a
 * scenario in FORCED mode takes the wave sub-step of step j from
 * f0 + (j/k)(f1 - f0) (E, H, D, DR clipped at 0), and at j = k its wave
 * action and roller energy are rescaled per cell to the forced E and DR, so
 * that the wave solver can take over; the others run the wave solver.  Dt,
 * boundaries, flow, sediment and means are the plain kernels throughout.
 * Does not synchronise.                                                    */
int  xbg_batch_forced_segment(xbg_batch* b, int k);
/* The judge: per scenario, the relative L2 distance ||pred - f|| / ||f||
 * of a prediction plane from the model's 2-D field f (XBG_F_*); pred: n
 * device plane pointers (NULL: scenario skipped, err = -1).  Synchronises. */
int  xbg_batch_rel_err(xbg_batch* b, int field, const void* const* pred,
                       double* err);

/* ---- no-allocation entry point ------------------------------------------
 * No counterpart in the reference.  For callers that may not allocate
 * device memory: a coupler or framework that owns the device through its
 * own pool allocator, or code that cannot afford the device-wide
 * synchronisation of cudaMalloc/cudaFree.  Computes, on `stream`, the flow
 * time-step candidate that xbg_compute_dt derives from the water depth:
 * *dt_out = 0.5 * min over cells of cfl*dx/sqrt(9.81*hh), with hh (nx*ny
 * values) and dt_out caller-owned device memory of the given precision.
 * It allocates nothing: its only scratch (per-block minima and a counter)
 * is a fixed XBG_NOALLOC_SCRATCH_BYTES array inside the library that every
 * GPU loading the library holds until exit.  Grids above
 * XBG_NOALLOC_MAX_CELLS cells return XBG_ERR_ARG.  All calls on a device
 * share that array, so calls that may overlap on the GPU race: order them.
 * The first call on a device looks the array's address up; make it before
 * any stream capture.  Does not synchronise.                              */
#define XBG_NOALLOC_MAX_BLOCKS     1184          /* 8 blocks x 148 SMs    */
#define XBG_NOALLOC_SCRATCH_BYTES  (256 + 8 * XBG_NOALLOC_MAX_BLOCKS)
#define XBG_NOALLOC_MAX_CELLS      (1LL << 30)
int  xbg_flow_dt_noalloc(int precision, const void* hh, int nx, int ny,
                         double dx, double cfl, void* dt_out, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* XBG_H */
