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


def test_model_from_input_files(tmp_path, monkeypatch):
    """A model set up from the reference's input files (.md bathymetry,
    sea-level and wind tables, an XBeach reuse boundary list) runs bit for
    bit like the same model set up from the arrays the files hold."""
    import math
    from xbeach_gpu_b200 import inputs
    monkeypatch.chdir(tmp_path)
    p, zb, bnd = make_case("linear_beach", nx=96, ny=48, ntheta=10)
    zb32 = zb.astype(np.float32).reshape(p.ny, p.nx)
    with open("bathy.md", "w") as f:
        f.write(f"{p.nx}\t{p.ny}\t{p.dx}\t0\t0\n")
        for j in range(p.ny):
            f.write(f"{j + 1}\t" + "\t".join(repr(float(v)) for v in zb32[j]) + "\n")
    open("wl.txt", "w").write("0\t0.1\t0.2\n100000\t0.1\t0.2\n")
    open("wind.txt", "w").write("# t spd dir\n0 5 270\n100000 5 270\n")
    dtbc = p.dtbc
    nrec = math.ceil(p.rtlength / dtbc)          # the records a reuse step holds
    bnd["q"][:nrec].astype("<f8").tofile("q0.bin")
    bnd["St"][:nrec].astype("<f8").tofile("E0.bin")
    open("list.txt", "w").write(f"{math.degrees(p.thetamin)} {math.degrees(p.thetamax)} "
                                f"{math.degrees(p.dtheta)} {dtbc} {p.rtlength}\n"
                                f"0.0 {bnd['Trep']} q0.bin E0.bin\n")
    a = Model(p, XBG_FP32)
    nx, ny, dx, ga, zbf = inputs.read_md("bathy.md")
    assert (nx, ny, dx) == (p.nx, p.ny, p.dx)
    inputs.apply_series(a, inputs.read_sealevel("wl.txt"), inputs.read_wind("wind.txt", ga))
    xb = inputs.XBeachReuse("list.txt")
    assert xb.nrec == nrec
    xb.apply(a, 0)
    a.init_state(zbf, 0.1, 0.2)
    b = Model(p, XBG_FP32)
    th = 1.5 * 3.14159265 - 0.0 - 270 * 3.14159265 / 180
    b.set_sealevel([0.0, 100000.0], [0.1, 0.1], [0.2, 0.2])
    b.set_wind([0.0, 100000.0], [5 * math.cos(th)] * 2, [5 * math.sin(th)] * 2)
    b.set_wave_boundary(0, bnd["St"][:nrec].astype(np.float32).astype(np.float64),
                        bnd["q"][:nrec].astype(np.float32).astype(np.float64), t0=0.0, tend=p.rtlength,
                        Trep=float(np.float32(bnd["Trep"])))
    b.init_state(zb32, 0.1, 0.2)
    a.advance(60)
    b.advance(60)
    for f in ("zs", "uu", "H", "ee", "zb"):
        np.testing.assert_array_equal(a.get(f), b.get(f), err_msg=f)
    a.close(); b.close()
