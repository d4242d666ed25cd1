"""Failure detection without a GPU fault.

The reference stops the process when its dt becomes NaN ("Model crashed!",
Wave_gpu.cu:642-647).  Here the dt pass checks the state on the device and a
non-finite water depth or level sets XBG_ERR_NAN in the handle's clock; the
status is sticky, every later step of that handle is skipped, and nothing
else is affected.  Failures are made on the host: a field poisoned with NaN
through xbg_set_field, and for the tensor-core kernels a bounded wait on a
barrier that nothing completes (XBG_NN_CHECK_TIMEOUT), after which the
kernel takes its time-out exit and the context stays usable.
"""
import numpy as np
import pytest

import pyoracle
from xbeach_gpu_b200.abi import XBG_FP32, XBG_FP64
from xbeach_gpu_b200.model import Batch, Model
from xbeach_gpu_b200.scenarios import make_case, make_ensemble

pytestmark = pytest.mark.gpu

XBG_ERR_NAN = 3
XBG_ERR_TIMEOUT = 5


def _beach(cls, precision=XBG_FP32):
    p, zb, bnd = make_case("linear_beach", nx=64, ny=32, ntheta=10)
    p.sedstart = 0.0
    h = cls(p, precision)
    h.set_wave_boundary(0, bnd["St"], bnd["q"], t0=0.0, tend=p.rtlength, Trep=bnd["Trep"])
    h.set_sealevel([0.0, 1e6], [0.0, 0.0], [0.0, 0.0])
    h.set_wind([0.0, 1e6], [0.0, 0.0], [0.0, 0.0])
    h.init_state(zb, 0.0, 0.0)
    return p, h


@pytest.mark.parametrize("precision", [XBG_FP32, XBG_FP64])
@pytest.mark.parametrize("field,value", [("hh", np.nan), ("zs", np.nan), ("zs", np.inf)])
def test_poisoned_state_sets_nan_status(field, value, precision):
    """A NaN or inf in hh or zs: the next step reports XBG_ERR_NAN (the step
    that found it is counted, as in the oracle), the time does not move, and
    later advances leave every field untouched.  The oracle, fed the same
    poisoned state, reports the same status."""
    p, m = _beach(Model, precision)
    m.advance(5)
    t0, dt0, n0, _, rc = m.time()
    assert rc == 0 and n0 == 5
    f = m.get(field)
    f[p.nx * 7 + 11] = value
    m.set(field, f)
    m.advance(3)
    t, dt, n, _, rc = m.time()
    assert rc == XBG_ERR_NAN
    assert (t, n) == (t0, n0 + 1)
    before = {k: m.get(k).copy() for k in ("ee", "uu", "zb", "H")}
    m.advance(10)
    t2, _, n2, _, rc2 = m.time()
    assert rc2 == XBG_ERR_NAN and (t2, n2) == (t0, n0 + 1)
    for k, v in before.items():
        assert np.array_equal(m.get(k), v, equal_nan=True), k
    m.close()
    # the oracle's dt logic makes the same call on the same state
    _, o = _beach(pyoracle.Oracle, precision)
    o.advance(5)
    g = o.get(field)
    g[p.nx * 7 + 11] = value
    o.set(field, g)
    assert o.L.xbgo_compute_dt(o.h) == XBG_ERR_NAN


def test_poisoned_scenario_goes_inactive_in_a_batch():
    """One scenario of a batch poisoned with NaN depth stops with XBG_ERR_NAN;
    the other scenarios go on and end bit for bit as in an unpoisoned batch."""
    sc = make_ensemble(4, seed=3, nx_range=(64, 160), ny_range=(32, 96), dtbc=5.0)

    def run(poison):
        b = Batch([p for p, _, _ in sc], XBG_FP32)
        for s, (p, zb, bnd) in enumerate(sc):
            m = b.scenario(s)
            m.set_wave_boundary(0, bnd["St"], bnd["q"], t0=0.0, tend=p.rtlength, Trep=bnd["Trep"])
            m.set_sealevel([0.0, 1e6], [0.0, 0.0], [0.0, 0.0])
            m.set_wind([0.0, 1e6], [0.0, 0.0], [0.0, 0.0])
            m.init_state(zb, 0.0, 0.0)
        b.advance(10)
        if poison:
            m = b.scenario(2)
            h = m.get("hh")
            h[h.size // 2] = np.nan
            m.set("hh", h)
        b.advance(20)
        st = b.status()
        out = {s: {f: b.scenario(s).get(f).copy() for f in ("zs", "uu", "H", "ee", "zb")} for s in range(len(sc))}
        b.close()
        return st, out

    st0, ref = run(False)
    st1, got = run(True)
    assert list(st0["status"]) == [0, 0, 0, 0] and list(st0["nstep"]) == [30] * 4
    assert list(st1["status"]) == [0, 0, XBG_ERR_NAN, 0]
    assert st1["nstep"][2] == 11 and st1["t"][2] < st0["t"][2]
    for s in (0, 1, 3):
        assert st1["nstep"][s] == 30 and st1["t"][s] == st0["t"][s]
        for f in ref[s]:
            assert np.array_equal(got[s][f], ref[s][f]), (s, f)


def test_tensor_core_wait_times_out_and_frees_tensor_memory():
    """XBG_NN_CHECK_TIMEOUT: every CTA of the GEMM waits, with a short limit,
    on a barrier that nothing completes; the launch records XBG_ERR_TIMEOUT,
    leaves C untouched, and frees its tensor memory, so that GEMMs launched
    afterwards on every SM (more CTAs than SMs) still allocate it and give
    the right product."""
    import torch
    from xbeach_gpu_b200 import surrogate as sg
    from xbeach_gpu_b200.surrogate import XBG_NN_CHECK_TIMEOUT
    L = sg.lib()
    g = torch.Generator(device="cuda").manual_seed(5)
    M, N, K = 128 * 400, 64, 128
    A = torch.randn(M, K, device="cuda", generator=g).bfloat16()
    B = torch.randn(N, K, device="cuda", generator=g).bfloat16()
    C = torch.full((M, N), 7.0, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    rc = L.xbg_nn_gemm(sg._p(A), sg._p(B), None, sg._p(C), M, N, K, K, K, N, XBG_NN_CHECK_TIMEOUT, 1, sg._p(err), None)
    assert rc == 0
    torch.cuda.synchronize()
    assert int(err.item()) == XBG_ERR_TIMEOUT
    assert bool((C == 7.0).all())
    for _ in range(2):
        err2 = sg.gemm(A, B, C)
        torch.cuda.synchronize()
        assert int(err2.item()) == 0
        ref = A.float() @ B.float().T
        assert torch.allclose(C, ref, rtol=1e-3, atol=1e-3 * ref.abs().max().item())
