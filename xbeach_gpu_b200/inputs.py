"""The reference's input files, read by the library (include/xbg_io.h):
bathymetry grids (.md, XBeach .dep), sea-level and wind series, wave-boundary
parameter series (constant records, JONSWAP records) and XBeach reuse
boundary files, with read_input.cpp's formats; plus the glue that hands them
to a Model (set_sealevel, set_wind, set_wave_boundary, init_state).
"""
import ctypes as C
import math

import numpy as np

from .model import _check, load

XBG_TAB_SEALEVEL, XBG_TAB_WIND, XBG_TAB_WAVECST, XBG_TAB_JONSWAP = 0, 1, 2, 3
TABLE_COLUMNS = {
    XBG_TAB_SEALEVEL: ("time", "wlev0", "wlev1"),
    XBG_TAB_WIND: ("time", "spd", "dir", "theta", "U", "V"),
    XBG_TAB_WAVECST: ("time", "Hs", "Tp", "Dp", "s"),
    XBG_TAB_JONSWAP: ("time", "Hs", "Tp", "Dp", "s", "gamma"),
}
_bound = False


def _lib():
    global _bound
    L = load()
    if not _bound:
        vp, ip, dp = C.c_void_p, C.c_int, C.POINTER(C.c_double)
        L.xbg_read_table.argtypes = [C.c_char_p, ip, C.c_double, C.c_double, dp, ip, C.POINTER(ip), C.POINTER(ip)]
        L.xbg_read_md_head.argtypes = [C.c_char_p, C.POINTER(ip), C.POINTER(ip), dp, dp]
        L.xbg_read_md.argtypes = [C.c_char_p, ip, ip, C.POINTER(C.c_float)]
        L.xbg_read_dep.argtypes = [C.c_char_p, ip, ip, C.POINTER(C.c_float)]
        L.xbg_read_xbbnd_head.argtypes = [C.c_char_p, dp]
        L.xbg_read_xbbnd_list.argtypes = [C.c_char_p, C.c_double, dp, dp, ip, C.POINTER(ip)]
        L.xbg_read_xbbnd_step.argtypes = [C.c_char_p, ip, ip, ip, ip, dp, dp, dp]
        L.xbg_read_spec_list.argtypes = [C.c_char_p, C.c_double, dp, C.c_char_p, ip, ip, C.POINTER(ip)]
        _bound = True
    return L


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def read_table(path, kind, grdalpha=0.0, rtlength=0.0):
    """A table file as an [nrec, ncol] float64 array (columns TABLE_COLUMNS[kind])."""
    L = _lib()
    n, nc = C.c_int(), C.c_int()
    _check(L.xbg_read_table(str(path).encode(), kind, grdalpha, rtlength, None, 0, C.byref(n), C.byref(nc)),
           f"read {path}")
    out = np.empty((n.value, nc.value), np.float64)
    _check(L.xbg_read_table(str(path).encode(), kind, grdalpha, rtlength, _dp(out), n.value, C.byref(n),
                            C.byref(nc)), f"read {path}")
    return out


def read_sealevel(path):
    return read_table(path, XBG_TAB_SEALEVEL)


def read_wind(path, grdalpha=0.0):
    return read_table(path, XBG_TAB_WIND, grdalpha)


def read_md(path):
    """A .md bathymetry: (nx, ny, dx, grdalpha [radians], zb [ny, nx] float32)."""
    L = _lib()
    nx, ny, dx, ga = C.c_int(), C.c_int(), C.c_double(), C.c_double()
    _check(L.xbg_read_md_head(str(path).encode(), C.byref(nx), C.byref(ny), C.byref(dx), C.byref(ga)),
           f"read {path}")
    zb = np.empty((ny.value, nx.value), np.float32)
    _check(L.xbg_read_md(str(path).encode(), nx.value, ny.value, zb.ctypes.data_as(C.POINTER(C.c_float))),
           f"read {path}")
    # the caller converts the grid rotation to radians (Wave_gpu.cu:1771)
    return nx.value, ny.value, dx.value, ga.value * math.pi / 180.0, zb


def read_dep(path, nx, ny):
    L = _lib()
    zb = np.empty((ny, nx), np.float32)
    _check(L.xbg_read_dep(str(path).encode(), nx, ny, zb.ctypes.data_as(C.POINTER(C.c_float))), f"read {path}")
    return zb


class XBeachReuse:
    """An XBeach reuse boundary list: header (thetamin, thetamax, dtheta in
    radians, dtbc, rtlength), entries (time, Trep, q file, E file) and the
    records of each entry."""

    def __init__(self, path):
        self.L = _lib()
        self.path = str(path)
        hdr = np.empty(5, np.float64)
        _check(self.L.xbg_read_xbbnd_head(self.path.encode(), _dp(hdr)), f"read {path}")
        self.thetamin, self.thetamax, self.dtheta, self.dtbc, self.rtlength = (float(x) for x in hdr)
        n = C.c_int()
        _check(self.L.xbg_read_xbbnd_list(self.path.encode(), self.rtlength, None, None, 0, C.byref(n)),
               f"read {path}")
        self.time = np.empty(n.value, np.float64)
        self.Trep = np.empty(n.value, np.float64)
        _check(self.L.xbg_read_xbbnd_list(self.path.encode(), self.rtlength, _dp(self.time), _dp(self.Trep),
                                          n.value, C.byref(n)), f"read {path}")
        self.nrec = int(math.ceil(self.rtlength / self.dtbc))

    def step(self, k, ny, ntheta):
        """(St [nrec, ntheta, ny], q [nrec, 4, ny], Trep) of entry k."""
        q = np.empty((self.nrec, 4, ny), np.float64)
        St = np.empty((self.nrec, ntheta, ny), np.float64)
        tr = C.c_double()
        _check(self.L.xbg_read_xbbnd_step(self.path.encode(), k, ny, ntheta, self.nrec, _dp(q), _dp(St),
                                          C.byref(tr)), f"read step {k} of {self.path}")
        return St, q, tr.value

    def apply(self, model, k, slot=0):
        """Hand entry k to the model as wave-boundary chunk `slot`."""
        St, q, tr = self.step(k, model.p.ny, model.p.ntheta)
        t0 = float(self.time[k])
        model.set_wave_boundary(slot, St, q, t0=t0, tend=t0 + self.rtlength, Trep=tr)


def apply_series(model, sealevel=None, wind=None):
    """Sea-level and wind tables (read_sealevel / read_wind) to the model."""
    if sealevel is not None:
        model.set_sealevel(sealevel[:, 0], sealevel[:, 1], sealevel[:, 2])
    if wind is not None:
        model.set_wind(wind[:, 0], wind[:, 4], wind[:, 5])


def read_spec_list(path, rtlength, name_len=1024):
    """ReadSPECBnd (read_input.cpp:534): the SWAN spectrum boundary list as
    (times [n], file names [n]) with the closing record rtlength after the
    last."""
    L = _lib()
    n = C.c_int()
    _check(L.xbg_read_spec_list(str(path).encode(), rtlength, None, None, 0, 0, C.byref(n)), f"read {path}")
    t = np.empty(n.value)
    buf = C.create_string_buffer(n.value * name_len)
    _check(L.xbg_read_spec_list(str(path).encode(), rtlength, _dp(t), buf, name_len, n.value, C.byref(n)),
           f"read {path}")
    raw = buf.raw
    names = [raw[k * name_len:(k + 1) * name_len].split(b"\0", 1)[0].decode() for k in range(n.value)]
    return t, names
