"""The library's netCDF writer (include/xbg_io.h) on the CPU: the file it
writes opens in an independent netCDF reader (scipy.io.netcdf_file) with the
reference's dimensions, variables, coordinate values and records
(writenetcdf.cpp:32-240); refusals on bad arguments and existing files."""
import os
import re

import numpy as np
import pytest

from xbeach_gpu_b200 import output

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_io_header_symbols_exported():
    from xbeach_gpu_b200 import build
    build.build(verbose=False)
    L = output._lib()
    txt = open(os.path.join(ROOT, "include", "xbg_io.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    syms = sorted(set(re.findall(r"\b(xbg_[a-z0-9_]+)\s*\(", txt)))
    assert set(syms) == {"xbg_nc_create", "xbg_nc_write_record", "xbg_nc_records", "xbg_nc_close",
                         "xbg_fetch_fields", "xbg_read_table", "xbg_read_md_head", "xbg_read_md",
                         "xbg_read_dep", "xbg_read_xbbnd_head", "xbg_read_xbbnd_list", "xbg_read_xbbnd_step",
                         "xbg_read_spec_list"}
    assert all(hasattr(L, s) for s in syms)


def _write(path, nx=7, ny=5, nt=3, nrec=3, seed=0, **kw):
    rng = np.random.default_rng(seed)
    dx, dth, tmin = 2.5, np.deg2rad(15.0), np.deg2rad(-22.5)
    f = output.NcFile(path, nx, ny, dx, nt, dth, tmin, ["zs", "H", "ee"], [3, 3, 4], **kw)
    recs = []
    for r in range(nrec):
        t = 12.5 * r + 0.1
        a = [rng.normal(size=ny * nx).astype(np.float32), rng.random(ny * nx).astype(np.float32),
             rng.random(nt * ny * nx).astype(np.float32)]
        f.write(t, a)
        recs.append((t, a))
        assert f.records() == r + 1
    f.close()
    return recs, (nx, ny, nt, dx, dth, tmin)


def test_roundtrip_in_an_independent_reader(tmp_path):
    from scipy.io import netcdf_file
    path = tmp_path / "out.nc"
    recs, (nx, ny, nt, dx, dth, tmin) = _write(path)
    raw = open(path, "rb").read(4)
    assert raw == b"CDF\x02"
    with netcdf_file(str(path), "r", mmap=False) as nc:
        assert nc.dimensions["xx"] == nx and nc.dimensions["yy"] == ny and nc.dimensions["theta"] == nt
        assert nc.dimensions["time"] is None          # the unlimited dimension
        v = nc.variables
        assert list(v) == ["time", "xx", "yy", "theta", "zs", "H", "ee"]
        assert v["zs"].dimensions == ("time", "yy", "xx")
        assert v["ee"].dimensions == ("time", "theta", "yy", "xx")
        for name in v:
            assert v[name].data.dtype == np.dtype(">f4"), name
        np.testing.assert_array_equal(v["xx"][:], (np.arange(nx) * dx).astype(np.float32))
        np.testing.assert_array_equal(v["yy"][:], (np.arange(ny) * dx).astype(np.float32))
        th = np.array([np.float32(t) * np.float32(dth) + np.float32(tmin) + np.float32(0.5) * np.float32(dth)
                       for t in range(nt)], dtype=np.float32)
        np.testing.assert_array_equal(v["theta"][:], th)
        assert v["time"].shape == (len(recs),)
        for r, (t, a) in enumerate(recs):
            assert v["time"][r] == np.float32(t)
            np.testing.assert_array_equal(v["zs"][r], a[0].reshape(ny, nx))
            np.testing.assert_array_equal(v["H"][r], a[1].reshape(ny, nx))
            np.testing.assert_array_equal(v["ee"][r], a[2].reshape(nt, ny, nx))


def test_no_records_and_large_grid_header(tmp_path):
    from scipy.io import netcdf_file
    path = tmp_path / "empty.nc"
    f = output.NcFile(path, 300, 200, 1.0, 18, 0.1, -0.9, [f"v{k}" for k in range(30)], [3] * 29 + [4])
    f.close()
    with netcdf_file(str(path), "r", mmap=False) as nc:
        assert nc.variables["v0"].shape == (0, 200, 300)
        assert nc.variables["v29"].shape == (0, 18, 200, 300)


def test_refusals(tmp_path):
    path = tmp_path / "a.nc"
    _write(path, nrec=1)
    with pytest.raises(Exception):
        _write(path, nrec=1)                      # NC_NOCLOBBER: an existing file is kept
    _write(path, nrec=2, clobber=True)
    with pytest.raises(Exception):
        output.NcFile(tmp_path / "b.nc", 4, 4, 1.0, 2, 0.1, 0.0, ["zs"], [2])   # ndims 3 or 4 only
    with pytest.raises(Exception):
        output.NcFile(tmp_path / "c.nc", 4, 4, 1.0, 2, 0.1, 0.0, ["xx"], [3])   # clashes with a coordinate
    with pytest.raises(Exception):
        output.NcFile(tmp_path / "d.nc", 4, 4, 1.0, 2, 0.1, 0.0, ["a", "a"], [3, 3])
    with pytest.raises(Exception):
        output.NcFile(tmp_path / "no_such_dir" / "e.nc", 4, 4, 1.0, 2, 0.1, 0.0, ["zs"], [3])
