/*
 * xbg_io.h -- host-side file IO around the B200-native XBeach_GPU step: the
 * model's map output as a netCDF file (written without libnetcdf) and the
 * reference's input files (bathymetry, sea level, wind, wave boundaries).
 *
 * The reference writes its map output with the netCDF-C library
 * (writenetcdf.cpp:32-240): creatncfileUD creates the file with the
 * dimensions xx (nx), yy (ny), theta (ntheta) and the unlimited time, and the
 * coordinate variables time, xx, yy, theta; defncvar adds one float variable
 * per requested output name, (time, yy, xx) for 2-D fields and
 * (time, theta, yy, xx) for the directional ones, and writes the initial
 * state as record 0; at every output time writenctimestep appends the time
 * and writencvarstep the record of each variable (Wave_gpu.cu:819-832,
 * 2943-2951).  The writer here produces the same dimensions, variables,
 * types and record layout in the netCDF classic format (64-bit offset
 * variant, "CDF\2"), encoded from the published format specification, so
 * any netCDF reader opens it.  All values are 32-bit floats, as in the
 * reference.
 *
 * Deviation, documented: the reference's theta axis is i*dtheta + 0.5*dtheta
 * because the thetamin it passes (the global at Wave_gpu.cu:110) is never
 * assigned; here the caller passes the model's thetamin, so the axis is the
 * bin centres.
 */
#ifndef XBG_IO_H
#define XBG_IO_H

#include <stddef.h>
#include <stdint.h>

#include "xbg.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct xbg_nc xbg_nc;

/* creatncfileUD + defncvar (writenetcdf.cpp:32-174) for all variables at
 * once.  names[k] / ndims[k] (3: time, yy, xx; 4: time, theta, yy, xx) for
 * k < nvars, names unique and not one of time, xx, yy, theta.  xx[i] = i*dx,
 * yy[j] = j*dx, theta[t] = t*dtheta + thetamin + dtheta/2 (floats).  An
 * existing file is an error unless clobber is 1 (the reference opens with
 * NC_NOCLOBBER).  No record is written yet.  XBG_ERR_IO on a file error. */
int xbg_nc_create(const char* path, int clobber, int nx, int ny, double dx,
                  int ntheta, double dtheta, double thetamin, int nvars,
                  const char* const* names, const int* ndims, xbg_nc** out);
/* writenctimestep + writencvarstep for every variable (writenetcdf.cpp:
 * 176-240): appends one record, time (stored as float) and data[k] with
 * nx*ny (ndims 3) or ntheta*nx*ny (ndims 4) floats in the model's layout
 * (i = ix + iy*nx, theta-planes outermost), then updates the record count
 * in the header, so the file is complete after every call. */
int xbg_nc_write_record(xbg_nc* f, double time, const float* const* data);
int xbg_nc_records(const xbg_nc* f, int64_t* nrec);
int xbg_nc_close(xbg_nc* f);

/* The asynchronous device-to-host copy of the output step (Wave_gpu.cu:
 * 823-831, a synchronous cudaMemcpy per variable there): enqueues one copy
 * per field on the handle's stream into host[k] (count of xbg_field_count
 * values of the handle's element type; pinned memory makes the copies
 * asynchronous) and returns without synchronising; xbg_sync (or any call
 * that returns host data) completes them.  ee, rr and zsold are taken from
 * the plane set current after the enqueued work. */
int xbg_fetch_fields(xbg_handle* h, const int* fields, int n, void* const* host);

/* ---- input files (read_input.cpp) -------------------------------------
 * The reference's file formats, read on the host.  Line-based files split
 * each line on tabs, or on spaces when a line has fewer values than the
 * format needs, or on commas (read_input.cpp:1476-1494); numbers parse like
 * std::stod.  A malformed file is XBG_ERR_FORMAT (the reference exits), a
 * file that does not open XBG_ERR_IO.  Angles in the files are degrees
 * nautical; grdalpha (grid rotation) is in radians.                        */
#define XBG_TAB_SEALEVEL 0  /* readWLfile (:259): time, wlev0, wlev1 (wlev1 =
                               wlev0 without a third column); '#' lines skipped */
#define XBG_TAB_WIND     1  /* readWNDfile (:332): time, spd, dir, theta, U, V
                               with theta = 1.5 pi - grdalpha - dir pi/180 and
                               (U, V) = spd (cos, sin) theta; '#' lines skipped */
#define XBG_TAB_WAVECST  2  /* ReadCstBnd (:407): time, Hs, Tp, Dp, s with Dp
                               = 1.5 pi - grdalpha - dir pi/180              */
#define XBG_TAB_JONSWAP  3  /* ReadJSWPBnd (:468): time, Hs, Tp, Dp, s, gamma,
                               plus a closing record at the last time + rtlength
                               with the last record's values                  */
/* Reads a table file of the given kind into out (row-major, *nrec records of
 * *ncol doubles).  out = NULL: only *nrec and *ncol; cap: records out holds. */
int xbg_read_table(const char* path, int kind, double grdalpha, double rtlength,
                   double* out, int cap, int* nrec, int* ncol);
/* readbathyHead (:1508): the first line of a .md bathymetry file, nx ny dx
 * (unused) grdalpha [degrees, as written].                                 */
int xbg_read_md_head(const char* path, int* nx, int* ny, double* dx,
                     double* grdalpha_deg);
/* readbathy (:1579): the .md grid, ny rows each led by its 1-based row number,
 * into zb[ix + (row-1)*nx] as floats; the header must give nx and ny.       */
int xbg_read_md(const char* path, int nx, int ny, float* zb);
/* readXBbathy (:1608): an XBeach .dep grid, nx*ny floats row by row.        */
int xbg_read_dep(const char* path, int nx, int ny, float* zb);
/* readXbbndhead (:25): the first line of an XBeach reuse boundary list:
 * hdr = thetamin, thetamax, dtheta [radians], dtbc, rtlength.              */
int xbg_read_xbbnd_head(const char* path, double* hdr);
/* readXbbndfile (:83): the list's entries (time, Trep) and a closing entry
 * rtlength after the last.  time = Trep = NULL: only *nrec.                */
int xbg_read_xbbnd_list(const char* path, double rtlength, double* time,
                        double* Trep, int cap, int* nrec);
/* readXbbndstep (:161): the records of entry `step`: its q file (4*ny*nrec
 * doubles, qbnd layout) and E file (ntheta*ny*nrec doubles, St layout), with
 * nrec = ceil(rtlength / dtbc), each value rounded to float as the
 * reference stores it, and the entry's Trep (float-rounded).  Directly the
 * St and qbnd of xbg_set_wave_boundary.                                    */
int xbg_read_xbbnd_step(const char* path, int step, int ny, int ntheta, int nrec,
                        double* q, double* St, double* Trep);

/* ReadSPECBnd (:534): a SWAN spectrum boundary list, one record per line
 * (time [s], spectrum file name), plus a closing record rtlength after the
 * last with the same file.  Names go NUL-terminated into rows of name_len
 * bytes of `names` (cap rows); a longer name is XBG_ERR_FORMAT.  time =
 * names = NULL: only *nrec.                                                */
int xbg_read_spec_list(const char* path, double rtlength, double* time,
                       char* names, int name_len, int cap, int* nrec);

#ifdef __cplusplus
}
#endif
#endif
