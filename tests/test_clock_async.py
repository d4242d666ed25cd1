"""The asynchronous clock read (xbg_get_time_async + xbg_clock_decode) gives,
once the stream has passed it, what the synchronous read gives at that
point of the stream: after every step of a run whose boundary records are
re-sent each step, and with the status word of a step that halted."""
import numpy as np
import pytest
import torch

from xbeach_gpu_b200.abi import XBG_CLOCK_BYTES, XBG_FP32
from xbeach_gpu_b200.model import Model
from xbeach_gpu_b200.scenarios import make_case

pytestmark = pytest.mark.gpu


def _model():
    p, zb, bnd = make_case("linear_beach", nx=64, ny=32, ntheta=6)
    m = Model(p, XBG_FP32)
    m.set_wave_boundary(0, bnd["St"], bnd["q"], t0=0.0, tend=p.rtlength, Trep=bnd["Trep"])
    m.set_sealevel([0.0, 1e6], [0.0, 0.0], [0.0, 0.0])
    m.set_wind([0.0, 1e6], [0.0, 0.0], [0.0, 0.0])
    m.init_state(zb, 0.0, 0.0)
    return p, m, bnd


def test_async_clock_read_matches_sync_read():
    p, m, bnd = _model()
    bufs = [torch.zeros(XBG_CLOCK_BYTES, dtype=torch.uint8, pin_memory=True) for _ in range(6)]
    stream = torch.cuda.ExternalStream(m.stream())
    ev = torch.cuda.Event()
    for k in range(6):
        m.step()
        m.time_async(bufs[k].data_ptr())
    ev.record(stream)
    ev.synchronize()
    got = [m.time_decode(b.data_ptr()) for b in bufs]
    t, dt, n, fl, rc = m.time()
    assert got[-1] == (t, dt, n, fl, rc)
    assert [g[2] for g in got] == list(range(1, 7)) and all(g[4] == 0 for g in got)
    assert all(got[k + 1][0] > got[k][0] for k in range(5))
    # a poisoned depth halts the next step; its copied clock carries the status
    hh = m.get("hh")
    hh[5] = np.nan
    m.set("hh", hh)
    m.step()
    m.time_async(bufs[0].data_ptr())
    ev.record(stream)
    ev.synchronize()
    assert m.time_decode(bufs[0].data_ptr())[4] == m.time()[4] != 0
    m.close()
