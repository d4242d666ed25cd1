"""Offshore wave-boundary records (include/xbg_bnd.h): wave groups and bound
long waves from a JONSWAP record (makjonswap + GenWGnLBW), or constant-wave
records (GenCstWave), as the St / q arrays Model.set_wave_boundary takes."""
import ctypes as C
import math

import numpy as np

from .abi import Params
from .model import _check, load

_bound = False


class WaveGen(C.Structure):
    """xbg_wavegen: one JONSWAP record and the generator's settings."""
    _fields_ = [("Hs", C.c_double), ("Tp", C.c_double), ("Dp", C.c_double), ("s", C.c_double),
                ("gamma", C.c_double), ("sprdthr", C.c_double), ("offdepth", C.c_double), ("nmax", C.c_double),
                ("fcutoff", C.c_double), ("nspr", C.c_int), ("seed", C.c_uint)]


def _lib():
    global _bound
    L = load()
    if not _bound:
        dp = C.POINTER(C.c_double)
        L.xbg_wavegen_default.argtypes = [C.POINTER(WaveGen)]
        L.xbg_wavegen_default.restype = None
        L.xbg_gen_wave_groups.argtypes = [C.POINTER(Params), C.POINTER(WaveGen), dp, dp, C.c_int, dp]
        L.xbg_gen_constant_waves.argtypes = [C.POINTER(Params), dp, C.c_int, dp, dp, dp, dp]
        _bound = True
    return L


def wavegen(**kw):
    L = _lib()
    w = WaveGen()
    L.xbg_wavegen_default(C.byref(w))
    for k, v in kw.items():
        setattr(w, k, v)
    return w


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def wave_groups(params, w):
    """(St [nrec, ntheta, ny], q [nrec, 4, ny], Trep) for one record."""
    L = _lib()
    nrec = int(math.ceil(params.rtlength / params.dtbc)) + 1
    St = np.empty((nrec, params.ntheta, params.ny), np.float64)
    q = np.empty((nrec, 4, params.ny), np.float64)
    tr = C.c_double()
    _check(L.xbg_gen_wave_groups(C.byref(params), C.byref(w), _dp(St), _dp(q), nrec, C.byref(tr)),
           "xbg_gen_wave_groups")
    return St, q, tr.value


def constant_waves(params, records, theta):
    """records [n, 5] = (time, Hs, Tp, Dp, s); theta: the bin directions."""
    L = _lib()
    rec = np.ascontiguousarray(records, np.float64)
    th = np.ascontiguousarray(theta, np.float64)
    n = rec.shape[0]
    St = np.empty((n, params.ntheta, params.ny), np.float64)
    q = np.empty((n, 4, params.ny), np.float64)
    Tp = np.empty(n, np.float64)
    _check(L.xbg_gen_constant_waves(C.byref(params), _dp(rec), n, _dp(th), _dp(St), _dp(q), _dp(Tp)),
           "xbg_gen_constant_waves")
    return St, q, Tp
