"""Map output of a model run as a netCDF file (include/xbg_io.h).

Mirrors the reference's output path: the output file is created with the
requested variables and the initial state as record 0 (creatncfileUD +
defncvar, Wave_gpu.cu:2943-2951); at every output time the running means are
divided by the step count, the time and every variable are appended as one
record, and the means restart (Wave_gpu.cu:784-930).  The device-to-host
copies of a record are enqueued together on the model's stream into pinned
host buffers (xbg_fetch_fields) and the record is written by the library's
classic-netCDF writer (xbg_nc_*), which needs no libnetcdf.

Output names are the reference's (read_input.cpp:1077).  Stored fields are
written as they are; kh = min(k hh, 10), sinh2kh = sinh(2 kh) and
wci = wci min(hh / hwci, 1) are formed from stored fields on the host.  The
reference's per-kernel temporaries (cgx, cgy, cx, cy, ctheta, sigm, dhdx,
dhdy, dudx, dudy, dvdx, dvdy, dzsdx, dzsdy, ududx, vdvdy, udvdx, vdudy) are
not kept by the fused kernels and are refused with a list of what is
available.
"""
import ctypes as C
import math

import numpy as np

from .abi import FIELD, FIELD_NAMES, INT_FIELDS, THETA_FIELDS, XBG_FLAG_ENDED, XBG_FLAG_OUTPUT_DUE
from .model import XbgError, _check, load

# read_input.cpp:1434: the variables written when the parameter file names none
DEFAULT_OUTVARS = ["zb", "zs", "uu", "vv", "H", "thetamean", "D", "urms", "ueu", "vev", "C", "dzb", "Fx",
                   "Fy", "hh", "Hmean", "uumean", "vvmean", "hhmean", "zsmean", "Cmean"]
DERIVED = {"kh": ("k", "hh"), "sinh2kh": ("k", "hh"), "wci": ("hh",)}
MAP_FIELDS = [n for n in FIELD_NAMES if n not in INT_FIELDS and n != "umeanbnd"]
NOT_KEPT = ["cgx", "cgy", "cx", "cy", "ctheta", "sigm", "dhdx", "dhdy", "dudx", "dudy", "dvdx", "dvdy",
            "dzsdx", "dzsdy", "ududx", "vdvdy", "udvdx", "vdudy"]

_bound = False


def _lib():
    global _bound
    L = load()
    if not _bound:
        vp, ip = C.c_void_p, C.c_int
        L.xbg_nc_create.argtypes = [C.c_char_p, ip, ip, ip, C.c_double, ip, C.c_double, C.c_double, ip,
                                    C.POINTER(C.c_char_p), C.POINTER(ip), C.POINTER(vp)]
        L.xbg_nc_write_record.argtypes = [vp, C.c_double, C.POINTER(vp)]
        L.xbg_nc_records.argtypes = [vp, C.POINTER(C.c_int64)]
        L.xbg_nc_close.argtypes = [vp]
        L.xbg_fetch_fields.argtypes = [vp, C.POINTER(ip), ip, C.POINTER(vp)]
        _bound = True
    return L


class NcFile:
    """The library's netCDF writer: dims xx, yy, theta, time; one float
    variable per name, (time, yy, xx) or (time, theta, yy, xx)."""

    def __init__(self, path, nx, ny, dx, ntheta, dtheta, thetamin, names, ndims, clobber=False):
        self.L = _lib()
        self.shapes = [(ny, nx) if d == 3 else (ntheta, ny, nx) for d in ndims]
        self.names = list(names)
        cn = (C.c_char_p * max(1, len(names)))(*[n.encode() for n in names])
        cd = (C.c_int * max(1, len(ndims)))(*ndims)
        self.f = C.c_void_p()
        _check(self.L.xbg_nc_create(str(path).encode(), 1 if clobber else 0, nx, ny, float(dx), ntheta,
                                    float(dtheta), float(thetamin), len(names), cn, cd, C.byref(self.f)),
               f"xbg_nc_create {path}")

    def write(self, time, arrays):
        bufs = []
        for a, shp in zip(arrays, self.shapes):
            a = np.ascontiguousarray(a, dtype=np.float32)
            if a.size != int(np.prod(shp)):
                raise ValueError(f"record of {a.size} values for a variable of shape {shp}")
            bufs.append(a)
        ptrs = (C.c_void_p * max(1, len(bufs)))(*[b.ctypes.data for b in bufs])
        _check(self.L.xbg_nc_write_record(self.f, float(time), ptrs), "xbg_nc_write_record")

    def records(self):
        n = C.c_int64()
        _check(self.L.xbg_nc_records(self.f, C.byref(n)), "xbg_nc_records")
        return n.value

    def close(self):
        if self.f:
            _check(self.L.xbg_nc_close(self.f), "xbg_nc_close")
            self.f = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class MapOutput:
    """The map output of one Model: `write()` appends a record of the
    current state at the current model time."""

    def __init__(self, model, path, outvars=None, clobber=False):
        import torch
        self.m = model
        p = model.p
        outvars = list(DEFAULT_OUTVARS if outvars is None else outvars)
        bad = [v for v in outvars if v not in MAP_FIELDS and v not in DERIVED]
        if bad:
            raise ValueError(f"output variables not available: {bad}; per-kernel temporaries of the "
                             f"reference ({', '.join(NOT_KEPT)}) are not kept; available: "
                             f"{MAP_FIELDS + sorted(DERIVED)}")
        self.outvars = outvars
        # fields to copy (stored ones, and the inputs of the derived ones)
        need = []
        for v in outvars:
            for f in (DERIVED[v] if v in DERIVED else (v,)):
                if f not in need:
                    need.append(f)
        self.fields = need
        self.host = {f: torch.empty(model.count(f), dtype=torch.float32 if model.dtype == np.float32
                                    else torch.float64, pin_memory=True) for f in need}
        ndims = [4 if v in THETA_FIELDS else 3 for v in outvars]
        self.nc = NcFile(path, p.nx, p.ny, p.dx, p.ntheta, p.dtheta, p.thetamin, outvars, ndims, clobber)
        self.L = _lib()

    def fetch(self):
        """Enqueue the copies of every needed field (no synchronisation)."""
        ids = (C.c_int * len(self.fields))(*[FIELD[f] for f in self.fields])
        dst = (C.c_void_p * len(self.fields))(*[self.host[f].data_ptr() for f in self.fields])
        _check(self.L.xbg_fetch_fields(self.m.h, ids, len(self.fields), dst), "xbg_fetch_fields")

    def _derived(self, v, a):
        p = self.m.p
        hh = a["hh"].astype(np.float64)
        if v == "wci":
            return p.wci * np.minimum(hh / p.hwci, 1.0)
        kh = np.minimum(a["k"].astype(np.float64) * hh, 10.0)
        return kh if v == "kh" else np.sinh(2.0 * kh)

    def write(self):
        t = self.m.time()[0]          # synchronises: the model's work is done
        self.fetch()
        self.m.sync()
        a = {f: self.host[f].numpy() for f in self.fields}
        self.nc.write(t, [self._derived(v, a) if v in DERIVED else a[v] for v in self.outvars])

    def close(self):
        self.nc.close()


def run(model, out, chunk=100, max_steps=None):
    """mainloopGPU with map output (Wave_gpu.cu:702-930): record 0 is the
    initial state; the model advances until an output time, where the means
    are divided by the step count, a record is written and the means restart;
    ends at endtime.  Returns the number of records written."""
    out.write()
    steps = 0
    n = 1
    while True:
        model.advance(chunk)
        steps += chunk
        t, dt, nstep, flags, rc = model.time()
        _check(rc, "advance")
        if flags & XBG_FLAG_OUTPUT_DUE:
            model.call("output_done")
            out.write()
            model.call("reset_means")
            n += 1
        if flags & XBG_FLAG_ENDED or (max_steps is not None and steps >= max_steps):
            return n
