"""The reference-side C++ binding of the integration guide, compiled and run.

tests/cxx/xbg_binding.cpp is the binding a maintainer adds to the reference's
host code (mainloop_xbg in place of mainloopGPU's device allocations and
step calls); the integration guide shows it verbatim, which the first test
checks.  It compiles against include/ and links libxbg_b200.so with g++
(no GPU needed); on a GPU the driver runs the reference's CPU-runnable case
for 20 s with map output every 10 s, and the file it writes must hold, bit
for bit, what the same calls made through the Python mirror give.
"""
import os
import re
import subprocess

import numpy as np
import pytest

from xbeach_gpu_b200.abi import XBG_FLAG_ENDED, XBG_FLAG_OUTPUT_DUE
from xbeach_gpu_b200.scenarios import make_case

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CXX = os.path.join(ROOT, "tests", "cxx")
LIBDIR = os.path.join(ROOT, "xbeach_gpu_b200")


def _compile(out_dir):
    from xbeach_gpu_b200 import build
    build.build(verbose=False)
    exe = os.path.join(out_dir, "xbg_driver")
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), "-I", CXX,
           os.path.join(CXX, "xbg_binding.cpp"), os.path.join(CXX, "driver.cpp"), "-L", LIBDIR, "-lxbg_b200",
           f"-Wl,-rpath,{LIBDIR}", "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_integration_guide_shows_the_compiled_binding():
    guide = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    blocks = re.findall(r"```c\+\+\n(.*?)```", guide, flags=re.S)
    src = open(os.path.join(CXX, "xbg_binding.cpp")).read()
    assert any(b == src for b in blocks), "INTEGRATION.md section 1 differs from tests/cxx/xbg_binding.cpp"


def test_binding_compiles_and_links(tmp_path):
    exe = _compile(str(tmp_path))
    assert os.path.exists(exe)


@pytest.mark.gpu
def test_binding_runs_the_reference_case(tmp_path):
    from scipy.io import netcdf_file
    from xbeach_gpu_b200.model import Model
    exe = _compile(str(tmp_path))
    p, zb, bnd = make_case("linear_beach")
    nrec = 64   # the records the 20 s run reaches (dtbc = 1 s), handed out as the chunk
    St, q = bnd["St"][:nrec], bnd["q"][:nrec]
    files = {}
    for name, arr, dt in (("zb", zb, np.float32), ("St", St, np.float64), ("q", q, np.float64)):
        files[name] = str(tmp_path / f"{name}.bin")
        np.ascontiguousarray(arr, dtype=dt).tofile(files[name])
    nc_path = str(tmp_path / "out.nc")
    r = subprocess.run([exe, files["zb"], files["St"], files["q"], str(nrec), "20", "10", nc_path],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    steps = int(r.stdout.strip().split("=")[1])
    # the same calls through the Python mirror
    p.endtime, p.outputtimestep = 20.0, 10.0
    m = Model(p)
    for slot in (0, 1):
        m.set_wave_boundary(slot, St, q, t0=3600.0 * slot, tend=3600.0 * (slot + 1), Trep=10.0 / 1.1)
    m.set_sealevel([0.0, 1e6], [0.0, 0.0], [0.0, 0.0])
    m.set_wind([0.0, 1e6], [0.0, 0.0], [0.0, 0.0])
    m.init_state(zb, 0.0, 0.0)
    records = []
    while True:
        m.advance(64)
        t, dt, n, fl, rc = m.time()
        assert rc == 0
        if fl & XBG_FLAG_OUTPUT_DUE:
            m.call("output_done")
            records.append((t, {f: m.get(f).copy() for f in ("zs", "uu", "H", "C", "Hmean", "ee")}))
            m.call("reset_means")
        if fl & XBG_FLAG_ENDED:
            break
    assert n == steps and len(records) == 2
    with netcdf_file(nc_path, "r", mmap=False) as f:
        tt = f.variables["time"][:].copy()
        assert tt.shape == (3,) and abs(tt[1] - 10.0) < 1e-3 and abs(tt[2] - 20.0) < 1e-3
        for k, (t, rec) in enumerate(records, start=1):
            for name, v in rec.items():
                got = f.variables[name][k].copy().ravel()
                assert np.array_equal(got, v.astype(np.float32)), (k, name)
