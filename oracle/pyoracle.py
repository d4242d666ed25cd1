"""TEST INFRASTRUCTURE ONLY: Python handles on the two CPU checkers.

  Oracle   -- oracle/_build/libxbg_oracle.so, the CPU restatement of the
              coupled step (FP32 or FP64), same call sequence as include/xbg.h
  RefEmu   -- oracle/_ref/libxbg_ref.so, the reference's own wave_CPU.cpp and
              CUDA kernel sources run on the CPU (built only where the
              reference checkout exists; the built library travels with the
              repository snapshot)

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module, as the checker of the CUDA path.
"""
import ctypes as C
import os
import subprocess

import numpy as np

from xbeach_gpu_b200.abi import (FIELD, INT_FIELDS, THETA_FIELDS, Params,
                                 XBG_FP32, XBG_FP64, STATUS_NAMES)

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "libxbg_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libxbg_ref.so")
_lib = None
_ref = None


def build(ref=True, ref_dir=None):
    """Compile the checkers (gcc).  The reference part is compiled in place
    from ref_dir (default: $XBG_REFERENCE) when that checkout exists; without
    one the prebuilt oracle/_ref libraries are used as they are."""
    subprocess.run(["make", "-s", "-C", HERE, "_build/libxbg_oracle.so"], check=True)
    ref_dir = ref_dir or os.environ.get("XBG_REFERENCE")
    if ref and ref_dir:
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF={ref_dir}"], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            build(ref=False)
        _lib = C.CDLL(ORACLE_SO)
        vp, ip, dp = C.c_void_p, C.c_int, C.POINTER(C.c_double)
        for name in ["compute_dt", "wave_boundary", "flow_boundary", "wave_step", "flow_step",
                     "sediment_step", "accumulate_means", "step", "output_done", "reset_means",
                     "destroy"]:
            getattr(_lib, "xbgo_" + name).argtypes = [vp]
        _lib.xbgo_create.argtypes = [C.POINTER(Params), ip, C.POINTER(vp)]
        _lib.xbgo_init_state.argtypes = [vp, vp, C.c_double, C.c_double]
        _lib.xbgo_field_count.argtypes = [vp, ip, C.POINTER(C.c_size_t)]
        _lib.xbgo_set_field.argtypes = [vp, ip, vp, C.c_size_t]
        _lib.xbgo_get_field.argtypes = [vp, ip, vp, C.c_size_t]
        _lib.xbgo_set_wave_boundary.argtypes = [vp, ip, vp, vp, ip, vp, C.c_double, C.c_double, C.c_double]
        _lib.xbgo_set_sealevel.argtypes = [vp, vp, vp, vp, ip]
        _lib.xbgo_set_wind.argtypes = [vp, vp, vp, vp, ip]
        _lib.xbgo_advance.argtypes = [vp, ip]
        _lib.xbgo_get_time.argtypes = [vp, dp, dp, C.POINTER(C.c_int64), C.POINTER(C.c_int)]
        _lib.xbgo_set_time.argtypes = [vp, C.c_double, C.c_double, C.c_double]
        _lib.xbgo_mass.argtypes = [vp, dp, dp, dp]
    return _lib


def ref_available():
    return os.path.exists(REF_SO)


def reflib():
    global _ref
    if _ref is None:
        if not os.path.exists(REF_SO):
            raise FileNotFoundError("oracle/_ref/libxbg_ref.so is not built (needs the reference checkout)")
        _ref = C.CDLL(REF_SO)
        vp, ip, fp = C.c_void_p, C.c_int, C.c_float
        _ref.xbgr_create.argtypes = [C.POINTER(Params), C.POINTER(vp)]
        for name in ["destroy", "wave_step", "flow_boundary", "flow_step", "sediment_step"]:
            getattr(_ref, "xbgr_" + name).argtypes = [vp]
        _ref.xbgr_set_field.argtypes = [vp, ip, vp, C.c_size_t]
        _ref.xbgr_get_field.argtypes = [vp, ip, vp, C.c_size_t]
        _ref.xbgr_set_step_inputs.argtypes = [vp, C.c_double, C.c_double, fp, vp, vp, vp, fp, fp, fp, fp, fp, fp]
    return _ref


def _check(rc, what):
    if rc != 0:
        raise RuntimeError(f"{what}: status {rc} ({STATUS_NAMES.get(rc, '?')})")


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p)


class Oracle:
    """CPU restatement with the same call sequence as the C ABI."""

    def __init__(self, params, precision=XBG_FP32):
        self.L = lib()
        self.p = params
        self.dtype = np.float32 if precision == XBG_FP32 else np.float64
        self.h = C.c_void_p()
        _check(self.L.xbgo_create(C.byref(params), precision, C.byref(self.h)), "xbgo_create")

    def __del__(self):
        if getattr(self, "h", None):
            self.L.xbgo_destroy(self.h)
            self.h = None

    def count(self, name):
        n = C.c_size_t()
        _check(self.L.xbgo_field_count(self.h, FIELD[name], C.byref(n)), "count")
        return n.value

    def set(self, name, arr):
        dt = np.int32 if name in INT_FIELDS else self.dtype
        a = np.ascontiguousarray(arr, dtype=dt).ravel()
        _check(self.L.xbgo_set_field(self.h, FIELD[name], _ptr(a), a.size), f"set {name}")

    def get(self, name):
        dt = np.int32 if name in INT_FIELDS else self.dtype
        a = np.empty(self.count(name), dtype=dt)
        _check(self.L.xbgo_get_field(self.h, FIELD[name], _ptr(a), a.size), f"get {name}")
        return a

    def init_state(self, zb, zs0=0.0, zs1=0.0):
        z = np.ascontiguousarray(zb, dtype=self.dtype).ravel()
        _check(self.L.xbgo_init_state(self.h, _ptr(z), zs0, zs1), "init_state")

    def set_wave_boundary(self, slot, St, q, times=None, t0=0.0, tend=0.0, Trep=10.0):
        St = np.ascontiguousarray(St, dtype=np.float64)
        q = np.ascontiguousarray(q, dtype=np.float64)
        nrec = St.shape[0]
        tp = None
        if times is not None:
            times = np.ascontiguousarray(times, dtype=np.float64)
            tp = _ptr(times)
        _check(self.L.xbgo_set_wave_boundary(self.h, slot, _ptr(St), _ptr(q), nrec, tp, t0, tend, Trep),
               "set_wave_boundary")

    def set_sealevel(self, t, w0, w1):
        t, w0, w1 = (np.ascontiguousarray(x, dtype=np.float64) for x in (t, w0, w1))
        _check(self.L.xbgo_set_sealevel(self.h, _ptr(t), _ptr(w0), _ptr(w1), t.size), "sealevel")

    def set_wind(self, t, u, v):
        t, u, v = (np.ascontiguousarray(x, dtype=np.float64) for x in (t, u, v))
        _check(self.L.xbgo_set_wind(self.h, _ptr(t), _ptr(u), _ptr(v), t.size), "wind")

    def call(self, name):
        _check(getattr(self.L, "xbgo_" + name)(self.h), name)

    def advance(self, n):
        _check(self.L.xbgo_advance(self.h, n), "advance")

    def time(self):
        t, dt, n, fl = C.c_double(), C.c_double(), C.c_int64(), C.c_int()
        rc = self.L.xbgo_get_time(self.h, C.byref(t), C.byref(dt), C.byref(n), C.byref(fl))
        return t.value, dt.value, n.value, fl.value, rc

    def set_time(self, t, dt, wdt):
        _check(self.L.xbgo_set_time(self.h, t, dt, wdt), "set_time")

    def mass(self):
        w, s, b = C.c_double(), C.c_double(), C.c_double()
        self.L.xbgo_mass(self.h, C.byref(w), C.byref(s), C.byref(b))
        return w.value, s.value, b.value


class RefEmu:
    """The reference's own CPU wave code and CUDA kernels, run on the CPU (FP32)."""

    def __init__(self, params):
        self.L = reflib()
        self.p = params
        self.h = C.c_void_p()
        _check(self.L.xbgr_create(C.byref(params), C.byref(self.h)), "xbgr_create")
        self.nx, self.ny, self.nt = params.nx, params.ny, params.ntheta

    def __del__(self):
        if getattr(self, "h", None):
            self.L.xbgr_destroy(self.h)
            self.h = None

    def _n(self, name):
        C_ = self.nx * self.ny
        if name in THETA_FIELDS:
            return C_ * self.nt
        if name == "umeanbnd":
            return self.ny
        return C_

    def set(self, name, arr):
        dt = np.int32 if name in INT_FIELDS else np.float32
        a = np.ascontiguousarray(arr, dtype=dt).ravel()
        _check(self.L.xbgr_set_field(self.h, FIELD[name], _ptr(a), a.size), f"set {name}")

    def get(self, name):
        dt = np.int32 if name in INT_FIELDS else np.float32
        a = np.empty(self._n(name), dtype=dt)
        _check(self.L.xbgr_set_field is not None and self.L.xbgr_get_field(self.h, FIELD[name], _ptr(a), a.size),
               f"get {name}")
        return a

    def step_inputs(self, dt, totaltime, Trep, St, qold, qnew, timesincelast, timenext,
                    zsbndi, zsbndn, windu=0.0, windv=0.0):
        St = np.ascontiguousarray(St, dtype=np.float32).ravel()
        qo = np.ascontiguousarray(qold, dtype=np.float32).ravel()
        qn = np.ascontiguousarray(qnew, dtype=np.float32).ravel()
        self._keep = (St, qo, qn)
        _check(self.L.xbgr_set_step_inputs(self.h, dt, totaltime, Trep, _ptr(St), _ptr(qo), _ptr(qn),
                                           timesincelast, timenext, zsbndi, zsbndn, windu, windv),
               "step_inputs")

    def call(self, name):
        _check(getattr(self.L, "xbgr_" + name)(self.h), name)
