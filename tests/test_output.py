"""Map output of a CUDA model run (xbeach_gpu_b200.output): record 0 is the
initial state, every later record is the state at an output time with the
running means divided by the step count (Wave_gpu.cu:784-930); each record
read back with an independent netCDF reader equals the fields read through
xbg_get_field at that time."""
import numpy as np
import pytest

from xbeach_gpu_b200 import output
from xbeach_gpu_b200.abi import XBG_FLAG_OUTPUT_DUE, XBG_FP32
from xbeach_gpu_b200.model import Model
from xbeach_gpu_b200.scenarios import make_case

pytestmark = pytest.mark.gpu

OUTVARS = output.DEFAULT_OUTVARS + ["ee", "k", "kh", "sinh2kh"]


def _model(endtime=None):
    p, zb, bnd = make_case("linear_beach", nx=96, ny=48, ntheta=10)
    p.outputtimestep = 3.0
    if endtime is not None:
        p.endtime = endtime
    m = Model(p, XBG_FP32)
    m.set_wave_boundary(0, bnd["St"], bnd["q"], t0=0.0, tend=p.rtlength, Trep=bnd["Trep"])
    m.set_sealevel([0.0, 1e6], [0.0, 0.0], [0.0, 0.0])
    m.set_wind([0.0, 1e6], [0.0, 0.0], [0.0, 0.0])
    m.init_state(zb, 0.0, 0.0)
    return p, m


def _expect(m, p, v):
    if v == "kh" or v == "sinh2kh":
        kh = np.minimum(m.get("k").astype(np.float64) * m.get("hh").astype(np.float64), 10.0)
        return (kh if v == "kh" else np.sinh(2 * kh)).astype(np.float32)
    return m.get(v).astype(np.float32)


def test_records_equal_the_fields_at_output_times(tmp_path):
    from scipy.io import netcdf_file
    p, m = _model()
    path = tmp_path / "map.nc"
    out = output.MapOutput(m, path, OUTVARS)
    out.write()                                   # record 0: the initial state
    want = [(m.time()[0], {v: _expect(m, p, v) for v in OUTVARS})]
    while len(want) < 4:
        m.advance(50)
        t, dt, n, flags, rc = m.time()
        assert rc == 0
        if flags & XBG_FLAG_OUTPUT_DUE:
            m.call("output_done")
            out.write()
            want.append((t, {v: _expect(m, p, v) for v in OUTVARS}))
            m.call("reset_means")
    out.close()
    with netcdf_file(str(path), "r", mmap=False) as nc:
        assert nc.variables["time"].shape == (len(want),)
        for r, (t, fields) in enumerate(want):
            assert nc.variables["time"][r] == np.float32(t)
            for v in OUTVARS:
                shape = (p.ntheta, p.ny, p.nx) if v == "ee" else (p.ny, p.nx)
                np.testing.assert_array_equal(nc.variables[v][r], fields[v].reshape(shape), err_msg=v)
        # the means of a later record are averages, not sums
        assert np.abs(nc.variables["zsmean"][2] - nc.variables["zs"][2]).max() < 0.5
    m.close()


def test_run_loop_writes_every_output_time(tmp_path):
    from scipy.io import netcdf_file
    p, m = _model(endtime=10.0)
    path = tmp_path / "run.nc"
    out = output.MapOutput(m, path)               # the reference's default variables
    n = output.run(m, out, chunk=40, max_steps=4000)
    out.close()
    with netcdf_file(str(path), "r", mmap=False) as nc:
        t = nc.variables["time"][:]
        assert len(t) == n == 4                   # t = 0, 3, 6, 9
        assert t[0] == 0.0 and np.allclose(t[1:], [3.0, 6.0, 9.0], atol=1e-4)


def test_refuses_temporaries(tmp_path):
    p, m = _model()
    with pytest.raises(ValueError, match="ctheta"):
        output.MapOutput(m, tmp_path / "x.nc", ["zs", "ctheta"])
    m.close()
