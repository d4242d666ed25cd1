"""Checkpoint / resume: a snapshot of the whole device state taken mid-run
and loaded into a fresh handle with the same parameters continues the run
bit for bit (fields, both ee/rr plane sets through the results, the clock),
in FP32 and FP64, with the TMA and the thread-copied rows passes; a snapshot
of another grid or precision is refused."""
import numpy as np
import pytest

from xbeach_gpu_b200.abi import FIELD_NAMES, XBG_FP32, XBG_FP64, XBG_PHASE_WAVE
from xbeach_gpu_b200.model import Model, XbgError
from xbeach_gpu_b200.scenarios import make_case

pytestmark = pytest.mark.gpu


def _model(precision, nx=96, ny=40, nt=8, boundary=True):
    p, zb, bnd = make_case("barred_beach", nx=nx, ny=ny, ntheta=nt)
    m = Model(p, precision)
    if boundary:
        m.set_wave_boundary(0, bnd["St"], bnd["q"], t0=0.0, tend=p.rtlength, Trep=bnd["Trep"])
        m.set_sealevel([0.0, 1e6], [0.0, 0.3], [0.0, 0.0])
        m.set_wind([0.0, 1e6], [0.0, 0.0], [0.0, 0.0])
        m.init_state(zb, 0.0, 0.0)
    return m


@pytest.mark.parametrize("variant", [1, 0])
@pytest.mark.parametrize("precision", [XBG_FP32, XBG_FP64])
def test_resume_from_snapshot_is_bit_identical(precision, variant):
    a = _model(precision)
    a.set_variant(XBG_PHASE_WAVE, variant)
    a.advance(17)
    snap = a.save_state()
    at_snap = a.time()
    a.advance(23)
    want = {f: a.get(f).copy() for f in FIELD_NAMES}
    want_t = a.time()
    # a fresh handle without any set-up of its own: the snapshot carries the
    # boundary slots, series and clock
    b = _model(precision, boundary=False)
    b.set_variant(XBG_PHASE_WAVE, variant)
    b.load_state(snap)
    assert b.time() == at_snap
    b.advance(23)
    assert b.time() == want_t
    for f in FIELD_NAMES:
        assert np.array_equal(b.get(f), want[f]), f
    a.close()
    b.close()


def test_snapshot_of_another_grid_or_precision_is_refused():
    a = _model(XBG_FP32)
    a.advance(3)
    snap = a.save_state()
    for other in (_model(XBG_FP64, boundary=False), _model(XBG_FP32, nx=100, boundary=False)):
        with pytest.raises(XbgError):
            other.load_state(snap)
        other.close()
    with pytest.raises(XbgError):
        a.load_state(snap[:-1])
    a.close()
