"""ctypes mirror of include/xbg.h: the parameter struct, field ids, status codes.

The reference keeps these as the XBGPUParam class (XBeachGPU.h:62-154) and as
~120 global device pointers (Wave_gpu.cu:26-241); the C ABI names each state
field by an enum value instead.
"""
import ctypes as C

XBG_OK = 0
XBG_ERR_ARG = 1
XBG_ERR_CUDA = 2
XBG_ERR_NAN = 3
XBG_ERR_DT = 4
XBG_ERR_TIMEOUT = 5
XBG_ERR_STATE = 6
XBG_ERR_NOMEM = 7
XBG_ERR_BOUNDARY = 8
STATUS_NAMES = {
    0: "ok", 1: "bad argument", 2: "CUDA error", 3: "model crashed (dt NaN/inf/0)",
    4: "initial dt too small", 5: "device wait timed out", 6: "call out of order",
    7: "out of device memory", 8: "ran past the uploaded wave boundary", 9: "file could not be opened or written",
    10: "input file format error",
}

XBG_FP32 = 0
XBG_FP64 = 1

XBG_PHASE_WAVE = 0   # xbg_set_kernel_variant phases
XBG_PHASE_FLOW = 1
XBG_PHASE_TILE = 2   # the pointwise passes' block shape: 0 32 x 8 cells, 1 64 x 4
XBG_CLOCK_BYTES = 240   # xbg_get_time_async copies this many bytes

XBG_FLAG_OUTPUT_DUE = 1
XBG_FLAG_ENDED = 2
XBG_FLAG_NEED_BOUNDARY = 4
XBG_FLAG_FALLBACK = 8

XBG_WAVE_PLAIN = 0      # xbg_batch_set_wave_mode
XBG_WAVE_FORCED = 1
XBG_WAVE_FALLBACK = 2

FIELD_NAMES = [
    "zb", "zs", "hh", "uu", "vv",
    "hu", "hv", "hum", "hvm", "qx", "qy",
    "ueu", "vev", "vmageu", "vmagev", "vu", "uv",
    "uuold", "vvold", "zsold", "dzsdt",
    "H", "E", "D", "DR", "R",
    "k", "c", "cg", "Fx", "Fy", "urms", "ust",
    "thetamean", "cfm", "fwm",
    "C", "ceqsg", "stdep", "dzb", "rolthick", "kturb",
    "Hmean", "uumean", "vvmean", "hhmean", "zsmean", "Cmean", "zsmax",
    "wetu", "wetv",
    "umeanbnd",
    "ee", "rr",
]
FIELD = {name: i for i, name in enumerate(FIELD_NAMES)}
INT_FIELDS = {"wetu", "wetv"}
THETA_FIELDS = {"ee", "rr"}


class Params(C.Structure):
    """xbg_params (include/xbg.h) == XBGPUParam (XBeachGPU.h:62-154)."""
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("dx", C.c_double),
        ("swave", C.c_int), ("flow", C.c_int), ("sedtrans", C.c_int), ("morphology", C.c_int),
        ("g", C.c_double), ("rho", C.c_double), ("eps", C.c_double),
        ("cf", C.c_double), ("cfsand", C.c_double), ("cfreef", C.c_double),
        ("nuh", C.c_double), ("nuhfac", C.c_double),
        ("usesmago", C.c_int),
        ("smag", C.c_double),
        ("lat", C.c_double), ("fc", C.c_double), ("Cd", C.c_double),
        ("wci", C.c_double), ("hwci", C.c_double),
        ("breakmodel", C.c_int),
        ("gammaa", C.c_double), ("n", C.c_double), ("alpha", C.c_double),
        ("gammax", C.c_double), ("beta", C.c_double),
        ("fw", C.c_double), ("fwsand", C.c_double), ("fwreef", C.c_double),
        ("roller", C.c_int),
        ("thetamin", C.c_double), ("thetamax", C.c_double), ("dtheta", C.c_double),
        ("ntheta", C.c_int),
        ("D50", C.c_double), ("D90", C.c_double), ("rhosed", C.c_double), ("wws", C.c_double),
        ("drydzmax", C.c_double), ("wetdzmax", C.c_double), ("maxslpchg", C.c_double),
        ("por", C.c_double), ("morfac", C.c_double), ("sus", C.c_double), ("bed", C.c_double),
        ("facsk", C.c_double), ("facas", C.c_double),
        ("wavebndtype", C.c_int),
        ("CFL", C.c_double), ("sedstart", C.c_double), ("outputtimestep", C.c_double),
        ("endtime", C.c_double),
        ("dtbc", C.c_double), ("rtlength", C.c_double),
        ("means", C.c_int),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


def default_params():
    """Python twin of xbg_params_default (XBeachGPU.h:62-154 defaults)."""
    import math
    p = Params()
    p.nx = 0; p.ny = 0; p.dx = 0.0
    p.swave = 1; p.flow = 1; p.sedtrans = 0; p.morphology = 0
    p.g = 9.81; p.rho = 1025.0; p.eps = 0.01
    p.cf = 0.01; p.cfsand = 0.0; p.cfreef = 0.0
    p.nuh = 1.0; p.nuhfac = 1.0; p.usesmago = 1; p.smag = 0.3
    p.lat = 0.0; p.fc = 0.0; p.Cd = 0.002; p.wci = 0.0; p.hwci = 0.1
    p.breakmodel = 1; p.gammaa = 0.6; p.n = 8.0; p.alpha = 1.0; p.gammax = 2.0; p.beta = 0.15
    p.fw = 0.001; p.fwsand = 0.0; p.fwreef = 0.0
    p.roller = 1
    p.thetamin = -90 * 3.14159265 / 180; p.thetamax = 90 * 3.14159265 / 180
    p.dtheta = 0.0; p.ntheta = 0
    p.D50 = 0.00038; p.D90 = 0.00053; p.rhosed = 2650.0; p.wws = 0.0509
    p.drydzmax = 1.0; p.wetdzmax = 0.3; p.maxslpchg = 0.01; p.por = 0.4; p.morfac = 1.0
    p.sus = 1.0; p.bed = 1.0; p.facsk = 0.2; p.facas = 0.2
    p.wavebndtype = 2
    p.CFL = 0.7; p.sedstart = 3600.0; p.outputtimestep = 0.0; p.endtime = 0.0
    p.dtbc = 1.0; p.rtlength = 3600.0
    p.means = 1
    _ = math
    return p


def sanity(p, endbnd):
    """Python twin of xbg_params_sanity: the step-path rules of checkparamsanity
    (read_input.cpp:1227-1443) plus the theta-bin count of waveinitGPU
    (Wavestep.cu:33-45) and the Coriolis parameter (Wave_gpu.cu:2060-2064)."""
    import math
    tiny = 0.0000001
    if p.nx <= 0 or p.ny <= 0 or p.dx < tiny:
        raise ValueError("nx, ny and dx must be set")
    if abs(p.endtime - 0.0) <= tiny:
        p.endtime = 1.0 / tiny
    p.endtime = min(p.endtime, endbnd)
    if p.swave == 0:
        p.ntheta = 1
        p.dtheta = p.thetamax - p.thetamin
    if abs(p.outputtimestep) <= tiny:
        p.outputtimestep = p.endtime
    if abs(p.cfsand) < tiny:
        if p.cf < tiny:
            p.cf = tiny
        p.cfsand = p.cf
    if abs(p.cfreef) < tiny:
        p.cfreef = p.cfsand
    if abs(p.fwsand) < tiny:
        if p.fw < tiny:
            p.fw = tiny
        p.fwsand = p.fw
    if abs(p.fwreef) < tiny:
        p.fwreef = p.fwsand
    if p.usesmago == 1:
        p.nuh = p.smag
    if p.swave == 1:
        if p.dtheta > 0.0:
            p.ntheta = int(round((p.thetamax - p.thetamin) / p.dtheta))
        else:
            if p.ntheta == 0:
                p.ntheta = 1
            p.dtheta = (p.thetamax - p.thetamin) / p.ntheta
    wearth = 3.14159265 * (1.0 / 24.0) / 1800.0
    p.fc = 2.0 * wearth * math.sin(p.lat)
    return p
