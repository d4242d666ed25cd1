"""Python handle on libxbg_b200.so, the CUDA implementation of the coupled step.

`Model` mirrors the reference's host step interface (XBeachGPU.h:348-353):
wavebnd -> wave_boundary, flowbnd -> flow_boundary, wavestep -> wave_step,
flowstep -> flow_step, sedimentstep -> sediment_step, plus the dt logic and
running means of mainloopGPU (compute_dt, accumulate_means) and whole graph-
replayed steps (step / advance).  Every call goes through the C ABI of
include/xbg.h; there is no other implementation behind it: if the library is
missing or no GPU is visible, construction raises.
"""
import ctypes as C
import os

import numpy as np

from .abi import FIELD, INT_FIELDS, Params, STATUS_NAMES, XBG_FP32

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libxbg_b200.so")
_lib = None

# Every entry point of include/xbg.h (checked by the tests against the header).
EXPORTS = [
    "xbg_params_default", "xbg_params_sanity", "xbg_create", "xbg_destroy", "xbg_status_string",
    "xbg_init_state", "xbg_field_count", "xbg_set_field", "xbg_get_field", "xbg_field_device_ptr",
    "xbg_set_wave_boundary", "xbg_set_sealevel", "xbg_set_wind", "xbg_compute_dt",
    "xbg_wave_boundary", "xbg_flow_boundary", "xbg_wave_step", "xbg_flow_step",
    "xbg_sediment_step", "xbg_accumulate_means", "xbg_step", "xbg_advance", "xbg_get_time",
    "xbg_get_time_async", "xbg_clock_decode", "xbg_state_bytes", "xbg_save_state", "xbg_load_state",
    "xbg_output_done", "xbg_reset_means", "xbg_set_time", "xbg_sync", "xbg_launch_count",
    "xbg_mass", "xbg_put_wave_records", "xbg_get_stream", "xbg_profile_step",
    "xbg_flow_dt_noalloc", "xbg_set_kernel_variant", "xbg_get_kernel_variant",
    "xbg_batch_create", "xbg_batch_destroy", "xbg_batch_scenario", "xbg_batch_advance", "xbg_batch_status",
    "xbg_batch_sync", "xbg_batch_get_stream", "xbg_batch_profile_step", "xbg_batch_set_grid",
    "xbg_batch_launch_count", "xbg_set_wave_forcing", "xbg_forcing_steps",
    "xbg_batch_set_kernel_variant", "xbg_batch_get_kernel_variant",
    "xbg_batch_set_wave_mode", "xbg_batch_set_forcing", "xbg_batch_forced_segment", "xbg_batch_rel_err",
]


class XbgError(RuntimeError):
    pass


def load():
    """Load the in-tree CUDA library (no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise XbgError(f"{LIB_PATH} is not built: run `python -m xbeach_gpu_b200.build`")
    L = C.CDLL(LIB_PATH)
    vp, ip, dp = C.c_void_p, C.c_int, C.POINTER(C.c_double)
    L.xbg_params_default.argtypes = [C.POINTER(Params)]
    L.xbg_params_default.restype = None
    L.xbg_params_sanity.argtypes = [C.POINTER(Params), C.c_double]
    L.xbg_create.argtypes = [C.POINTER(Params), ip, C.POINTER(vp)]
    L.xbg_status_string.argtypes = [ip]
    L.xbg_status_string.restype = C.c_char_p
    for n in ["destroy", "compute_dt", "wave_boundary", "flow_boundary", "wave_step", "flow_step",
              "sediment_step", "accumulate_means", "step", "output_done", "reset_means", "sync"]:
        getattr(L, "xbg_" + n).argtypes = [vp]
    L.xbg_init_state.argtypes = [vp, vp, C.c_double, C.c_double]
    L.xbg_field_count.argtypes = [vp, ip, C.POINTER(C.c_size_t)]
    L.xbg_set_field.argtypes = [vp, ip, vp, C.c_size_t]
    L.xbg_get_field.argtypes = [vp, ip, vp, C.c_size_t]
    L.xbg_field_device_ptr.argtypes = [vp, ip, C.POINTER(vp), C.POINTER(C.c_size_t)]
    L.xbg_set_wave_boundary.argtypes = [vp, ip, vp, vp, ip, vp, C.c_double, C.c_double, C.c_double]
    L.xbg_set_sealevel.argtypes = [vp, vp, vp, vp, ip]
    L.xbg_set_wind.argtypes = [vp, vp, vp, vp, ip]
    L.xbg_advance.argtypes = [vp, ip]
    L.xbg_get_time.argtypes = [vp, dp, dp, C.POINTER(C.c_int64), C.POINTER(C.c_int)]
    L.xbg_get_time_async.argtypes = [vp, vp]
    L.xbg_clock_decode.argtypes = [vp, vp, dp, dp, C.POINTER(C.c_int64), C.POINTER(C.c_int)]
    L.xbg_state_bytes.argtypes = [vp, C.POINTER(C.c_size_t)]
    L.xbg_save_state.argtypes = [vp, vp, C.c_size_t]
    L.xbg_load_state.argtypes = [vp, vp, C.c_size_t]
    L.xbg_set_time.argtypes = [vp, C.c_double, C.c_double, C.c_double]
    L.xbg_launch_count.argtypes = [vp, C.POINTER(C.c_int64)]
    L.xbg_mass.argtypes = [vp, dp, dp, dp]
    L.xbg_put_wave_records.argtypes = [vp, ip, ip, ip, vp, vp]
    L.xbg_get_stream.argtypes = [vp, C.POINTER(vp)]
    L.xbg_profile_step.argtypes = [vp, C.POINTER(C.c_float), C.POINTER(C.c_char_p), C.POINTER(ip)]
    L.xbg_flow_dt_noalloc.argtypes = [ip, vp, ip, ip, C.c_double, C.c_double, vp, vp]
    L.xbg_set_kernel_variant.argtypes = [vp, ip, ip]
    L.xbg_get_kernel_variant.argtypes = [vp, ip, C.POINTER(ip)]
    L.xbg_set_wave_forcing.argtypes = [vp, C.POINTER(vp), C.POINTER(vp), C.c_double, ip]
    L.xbg_forcing_steps.argtypes = [vp, C.POINTER(vp), C.POINTER(vp), ip]
    L.xbg_batch_create.argtypes = [C.POINTER(Params), ip, ip, C.POINTER(vp)]
    L.xbg_batch_destroy.argtypes = [vp]
    L.xbg_batch_scenario.argtypes = [vp, ip, C.POINTER(vp)]
    L.xbg_batch_advance.argtypes = [vp, ip]
    L.xbg_batch_status.argtypes = [vp, vp, vp, vp, vp, vp]
    L.xbg_batch_sync.argtypes = [vp]
    L.xbg_batch_get_stream.argtypes = [vp, C.POINTER(vp)]
    L.xbg_batch_profile_step.argtypes = [vp, C.POINTER(C.c_float), C.POINTER(C.c_char_p), C.POINTER(ip)]
    L.xbg_batch_set_grid.argtypes = [vp, ip, ip]
    L.xbg_batch_launch_count.argtypes = [vp, C.POINTER(C.c_int64)]
    L.xbg_batch_set_wave_mode.argtypes = [vp, ip, ip]
    L.xbg_batch_set_kernel_variant.argtypes = [vp, ip, ip]
    L.xbg_batch_get_kernel_variant.argtypes = [vp, ip, C.POINTER(ip)]
    L.xbg_batch_set_forcing.argtypes = [vp, ip, C.POINTER(vp), C.POINTER(vp)]
    L.xbg_batch_forced_segment.argtypes = [vp, ip]
    L.xbg_batch_rel_err.argtypes = [vp, ip, C.POINTER(vp), vp]
    _lib = L
    return L


def _check(rc, what):
    if rc != 0:
        raise XbgError(f"{what}: status {rc} ({STATUS_NAMES.get(rc, '?')})")


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p)


class Model:
    """One device-resident model (one xbg_handle)."""

    def __init__(self, params, precision=XBG_FP32, _handle=None):
        self.L = load()
        self.p = params
        self.dtype = np.float32 if precision == XBG_FP32 else np.float64
        self.owned = _handle is None
        if _handle is not None:   # a batch's scenario: the batch frees it
            self.h = _handle
            return
        self.h = C.c_void_p()
        _check(self.L.xbg_create(C.byref(params), precision, C.byref(self.h)), "xbg_create")

    def close(self):
        if getattr(self, "h", None):
            if self.owned:
                self.L.xbg_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def count(self, name):
        n = C.c_size_t()
        _check(self.L.xbg_field_count(self.h, FIELD[name], C.byref(n)), "count")
        return n.value

    def set(self, name, arr):
        dt = np.int32 if name in INT_FIELDS else self.dtype
        a = np.ascontiguousarray(arr, dtype=dt).ravel()
        _check(self.L.xbg_set_field(self.h, FIELD[name], _ptr(a), a.size), f"set {name}")

    def get(self, name, out=None):
        dt = np.int32 if name in INT_FIELDS else self.dtype
        a = out if out is not None else np.empty(self.count(name), dtype=dt)
        _check(self.L.xbg_get_field(self.h, FIELD[name], _ptr(a), a.size), f"get {name}")
        return a

    def device_ptr(self, name):
        p, n = C.c_void_p(), C.c_size_t()
        _check(self.L.xbg_field_device_ptr(self.h, FIELD[name], C.byref(p), C.byref(n)), "device_ptr")
        return p.value, n.value

    def init_state(self, zb, zs0=0.0, zs1=0.0):
        z = np.ascontiguousarray(zb, dtype=self.dtype).ravel()
        _check(self.L.xbg_init_state(self.h, _ptr(z), zs0, zs1), "init_state")

    def set_wave_boundary(self, slot, St, q, times=None, t0=0.0, tend=0.0, Trep=10.0):
        St = np.ascontiguousarray(St, dtype=np.float64)
        q = np.ascontiguousarray(q, dtype=np.float64)
        tp = None
        if times is not None:
            times = np.ascontiguousarray(times, dtype=np.float64)
            tp = _ptr(times)
        _check(self.L.xbg_set_wave_boundary(self.h, slot, _ptr(St), _ptr(q), St.shape[0], tp, t0, tend, Trep),
               "set_wave_boundary")

    def set_sealevel(self, t, w0, w1):
        t, w0, w1 = (np.ascontiguousarray(x, dtype=np.float64) for x in (t, w0, w1))
        _check(self.L.xbg_set_sealevel(self.h, _ptr(t), _ptr(w0), _ptr(w1), t.size), "sealevel")

    def set_wind(self, t, u, v):
        t, u, v = (np.ascontiguousarray(x, dtype=np.float64) for x in (t, u, v))
        _check(self.L.xbg_set_wind(self.h, _ptr(t), _ptr(u), _ptr(v), t.size), "wind")

    def call(self, name):
        _check(getattr(self.L, "xbg_" + name)(self.h), name)

    # the reference's step names
    def compute_dt(self): self.call("compute_dt")
    def wave_boundary(self): self.call("wave_boundary")
    def flow_boundary(self): self.call("flow_boundary")
    def wave_step(self): self.call("wave_step")
    def flow_step(self): self.call("flow_step")
    def sediment_step(self): self.call("sediment_step")
    def accumulate_means(self): self.call("accumulate_means")

    def step(self):
        self.call("step")

    def advance(self, n):
        _check(self.L.xbg_advance(self.h, n), "advance")

    def sync(self):
        self.call("sync")

    def time(self):
        t, dt, n, fl = C.c_double(), C.c_double(), C.c_int64(), C.c_int()
        rc = self.L.xbg_get_time(self.h, C.byref(t), C.byref(dt), C.byref(n), C.byref(fl))
        return t.value, dt.value, n.value, fl.value, rc

    def time_async(self, buf):
        """Enqueue a copy of the device clock into buf (XBG_CLOCK_BYTES of
        pinned host memory, e.g. a pinned uint8 torch tensor's data_ptr()) in
        the model's stream order; read it with time_decode once the stream
        has passed it."""
        _check(self.L.xbg_get_time_async(self.h, C.c_void_p(buf)), "get_time_async")

    def time_decode(self, buf):
        """(t, dt, nstep, flags, status) from a clock copied by time_async."""
        t, dt, n, fl = C.c_double(), C.c_double(), C.c_int64(), C.c_int()
        rc = self.L.xbg_clock_decode(self.h, C.c_void_p(buf), C.byref(t), C.byref(dt), C.byref(n), C.byref(fl))
        return t.value, dt.value, n.value, fl.value, rc

    def save_state(self):
        """A snapshot of the whole device state (numpy uint8 array); see
        load_state."""
        n = C.c_size_t()
        _check(self.L.xbg_state_bytes(self.h, C.byref(n)), "state_bytes")
        buf = np.empty(n.value, np.uint8)
        _check(self.L.xbg_save_state(self.h, buf.ctypes.data_as(C.c_void_p), n.value), "save_state")
        return buf

    def load_state(self, buf):
        """Restore a snapshot taken by save_state on a handle with the same
        parameters: the run continues from it bit for bit."""
        buf = np.ascontiguousarray(buf, dtype=np.uint8)
        _check(self.L.xbg_load_state(self.h, buf.ctypes.data_as(C.c_void_p), buf.size), "load_state")

    def set_time(self, t, dt, wdt):
        _check(self.L.xbg_set_time(self.h, t, dt, wdt), "set_time")

    def launches(self):
        n = C.c_int64()
        _check(self.L.xbg_launch_count(self.h, C.byref(n)), "launch_count")
        return n.value

    def put_wave_records(self, slot, first, St, q):
        """Stream records into a chunk (no synchronisation); St/q must stay
        alive until the stream has consumed them (pinned memory for overlap)."""
        _check(self.L.xbg_put_wave_records(self.h, slot, first, St.shape[0], _ptr(St), _ptr(q)),
               "put_wave_records")

    def stream(self):
        s = C.c_void_p()
        _check(self.L.xbg_get_stream(self.h, C.byref(s)), "get_stream")
        return s.value

    def set_wave_forcing(self, f0, f1, w, rescale=False):
        """E, H, D, DR, Fx, Fy = f0 + w (f1 - f0); f0, f1: six device plane
        pointers (ints) each."""
        a = (C.c_void_p * 6)(*[C.c_void_p(int(x)) for x in f0])
        b = (C.c_void_p * 6)(*[C.c_void_p(int(x)) for x in f1])
        _check(self.L.xbg_set_wave_forcing(self.h, a, b, float(w), 1 if rescale else 0), "set_wave_forcing")

    def forcing_steps(self, f0, f1, k):
        """k coupled steps with the wave sub-step replaced by the forcing
        f0 + (j/k)(f1 - f0), rescaled at j = k (one CUDA graph per (f0, f1, k));
        f0, f1: six device plane pointers (ints) each."""
        a = (C.c_void_p * 6)(*[C.c_void_p(int(x)) for x in f0])
        b = (C.c_void_p * 6)(*[C.c_void_p(int(x)) for x in f1])
        _check(self.L.xbg_forcing_steps(self.h, a, b, int(k)), "forcing_steps")

    def profile_step(self):
        """One non-graph step with an event after every kernel: [(name, ms)]."""
        cap = 64
        ms = (C.c_float * cap)()
        names = (C.c_char_p * cap)()
        n = C.c_int(cap)
        _check(self.L.xbg_profile_step(self.h, ms, names, C.byref(n)), "profile_step")
        return [(names[k].decode(), float(ms[k])) for k in range(n.value)]

    def set_variant(self, phase, variant):
        """Kernel variant of a phase (XBG_PHASE_WAVE: 1 / 2 TMA tiles with one /
        two cells per thread, 0 thread-copied tiles; XBG_PHASE_FLOW: 1 fused
        momentum pass, 0 two passes; XBG_PHASE_TILE: the pointwise passes in
        0 32 x 8 or 1 64 x 4 blocks)."""
        _check(self.L.xbg_set_kernel_variant(self.h, phase, variant), "set_kernel_variant")

    def variant(self, phase):
        v = C.c_int()
        _check(self.L.xbg_get_kernel_variant(self.h, phase, C.byref(v)), "get_kernel_variant")
        return v.value

    def mass(self):
        w, s, b = C.c_double(), C.c_double(), C.c_double()
        _check(self.L.xbg_mass(self.h, C.byref(w), C.byref(s), C.byref(b)), "mass")
        return w.value, s.value, b.value


class Batch:
    """n scenarios advanced together, one launch per kernel for all of them
    (xbg_batch_*).  batch.scenario(s) is a Model on the batch's handle s for
    fields, boundaries and time; advance() steps all of them."""

    def __init__(self, params_list, precision=XBG_FP32):
        self.L = load()
        self.n = len(params_list)
        arr = (Params * self.n)(*params_list)
        self.b = C.c_void_p()
        _check(self.L.xbg_batch_create(arr, self.n, precision, C.byref(self.b)), "xbg_batch_create")
        self.models = []
        for s, p in enumerate(params_list):
            h = C.c_void_p()
            _check(self.L.xbg_batch_scenario(self.b, s, C.byref(h)), "xbg_batch_scenario")
            self.models.append(Model(p, precision, _handle=h))

    def scenario(self, s):
        return self.models[s]

    def advance(self, nsteps):
        _check(self.L.xbg_batch_advance(self.b, nsteps), "xbg_batch_advance")

    def sync(self):
        _check(self.L.xbg_batch_sync(self.b), "xbg_batch_sync")

    def status(self):
        n = self.n
        t, dt = np.zeros(n), np.zeros(n)
        ns = np.zeros(n, np.int64)
        fl, st = np.zeros(n, np.int32), np.zeros(n, np.int32)
        _check(self.L.xbg_batch_status(self.b, _ptr(t), _ptr(dt), _ptr(ns), _ptr(fl), _ptr(st)), "xbg_batch_status")
        return dict(t=t, dt=dt, nstep=ns, flags=fl, status=st)

    def stream(self):
        s = C.c_void_p()
        _check(self.L.xbg_batch_get_stream(self.b, C.byref(s)), "xbg_batch_get_stream")
        return s.value

    def set_grid(self, shape, blocks):
        _check(self.L.xbg_batch_set_grid(self.b, shape, blocks), "xbg_batch_set_grid")

    def launches(self):
        n = C.c_int64()
        _check(self.L.xbg_batch_launch_count(self.b, C.byref(n)), "xbg_batch_launch_count")
        return n.value

    def set_variant(self, phase, variant):
        _check(self.L.xbg_batch_set_kernel_variant(self.b, phase, variant), "xbg_batch_set_kernel_variant")

    def variant(self, phase):
        v = C.c_int()
        _check(self.L.xbg_batch_get_kernel_variant(self.b, phase, C.byref(v)), "xbg_batch_get_kernel_variant")
        return v.value

    def set_wave_mode(self, s, mode):
        """XBG_WAVE_PLAIN / XBG_WAVE_FORCED / XBG_WAVE_FALLBACK for scenario s."""
        _check(self.L.xbg_batch_set_wave_mode(self.b, s, mode), "xbg_batch_set_wave_mode")

    def set_forcing(self, s, f0, f1):
        """Scenario s's forcing planes (six device pointers each, E H D DR Fx Fy)."""
        a = (C.c_void_p * 6)(*[C.c_void_p(int(x)) for x in f0])
        b = (C.c_void_p * 6)(*[C.c_void_p(int(x)) for x in f1])
        _check(self.L.xbg_batch_set_forcing(self.b, s, a, b), "xbg_batch_set_forcing")

    def forced_segment(self, k):
        """k steps; forced scenarios take their wave sub-step from the forcing."""
        _check(self.L.xbg_batch_forced_segment(self.b, int(k)), "xbg_batch_forced_segment")

    def rel_err(self, field, preds):
        """Per scenario ||pred - field|| / ||field|| (preds: device pointers or None)."""
        arr = (C.c_void_p * self.n)(*[C.c_void_p(int(x)) if x else None for x in preds])
        out = np.zeros(self.n)
        _check(self.L.xbg_batch_rel_err(self.b, FIELD[field], arr, _ptr(out)), "xbg_batch_rel_err")
        return out

    def profile_step(self):
        cap = 64
        ms = (C.c_float * cap)()
        names = (C.c_char_p * cap)()
        n = C.c_int(cap)
        _check(self.L.xbg_batch_profile_step(self.b, ms, names, C.byref(n)), "xbg_batch_profile_step")
        return [(names[k].decode(), ms[k]) for k in range(n.value)]

    def close(self):
        if getattr(self, "b", None):
            for m in self.models:
                m.h = None
            self.L.xbg_batch_destroy(self.b)
            self.b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
