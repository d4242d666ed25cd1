"""The library's input-file readers (include/xbg_io.h) against the
reference's own readers (read_input.cpp, compiled in place into
oracle/_ref/libxbg_ref_io.so with plain-C entry points): seeded files in the
reference's formats, with tab, space and comma separators, comment lines and
trailing text, read by both; results bit for bit equal.  Malformed files:
the library returns XBG_ERR_FORMAT where the reference exits."""
import ctypes as C
import math
import os

import numpy as np
import pytest

from xbeach_gpu_b200 import inputs

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_IO = os.path.join(ROOT, "oracle", "_ref", "libxbg_ref_io.so")


@pytest.fixture(scope="module")
def ref():
    if not os.path.exists(REF_IO):
        pytest.skip("oracle/_ref/libxbg_ref_io.so not built (needs the reference checkout)")
    L = C.CDLL(REF_IO)
    dp, ip = C.POINTER(C.c_double), C.c_int
    L.ref_io_sealevel.argtypes = [C.c_char_p, dp, ip]
    L.ref_io_wind.argtypes = [C.c_char_p, C.c_double, dp, ip]
    L.ref_io_wave.argtypes = [C.c_char_p, ip, C.c_double, C.c_double, dp, ip]
    L.ref_io_md_head.argtypes = [C.c_char_p, C.POINTER(ip), C.POINTER(ip), dp, dp]
    L.ref_io_md.argtypes = [C.c_char_p, C.POINTER(C.c_float)]
    L.ref_io_dep.argtypes = [C.c_char_p, ip, ip, C.POINTER(C.c_float)]
    L.ref_io_xbhead.argtypes = [C.c_char_p, dp]
    L.ref_io_xblist.argtypes = [C.c_char_p, C.c_double, dp, dp, ip]
    L.ref_io_xbstep.argtypes = [C.c_char_p, C.c_double, C.c_double, ip, ip, ip, ip, dp, dp, dp]
    L.ref_io_speclist.argtypes = [C.c_char_p, C.c_double, dp, C.c_char_p, ip, ip]
    return L


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _num(rng):
    v = rng.normal() * 10.0 ** int(rng.integers(-3, 4))
    return rng.choice([f"{v:.6f}", f"{v:.17g}", f"{v:e}", f"{v:.3f}"])


def _table_file(path, rng, ncol, comments, nrows=40):
    lines = []
    for r in range(nrows):
        sep = rng.choice(["\t", " ", ",", "  ", "\t\t"])
        vals = [f"{r * 3.6 + rng.random():.4f}"] + [_num(rng) for _ in range(ncol - 1)]
        line = sep.join(vals)
        if rng.random() < 0.2:
            line += sep                   # trailing separator
        lines.append(line)
        if comments and rng.random() < 0.15:
            lines.append("# a comment line")
        if rng.random() < 0.1:
            lines.append("")
    open(path, "w").write("\n".join(lines) + "\n")


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_sealevel_and_wind_tables(ref, tmp_path, seed):
    rng = np.random.default_rng(seed)
    for ncol in (2, 3):
        f = str(tmp_path / f"wl{ncol}.txt")
        _table_file(f, rng, ncol, comments=True)
        ours = inputs.read_sealevel(f)
        want = np.empty_like(ours)
        n = ref.ref_io_sealevel(f.encode(), _dp(want), len(want))
        assert n == len(ours)
        np.testing.assert_array_equal(ours, want)
    f = str(tmp_path / "wind.txt")
    _table_file(f, rng, 3, comments=True)
    ga = 0.3 * seed
    ours = inputs.read_wind(f, ga)
    want = np.empty_like(ours)
    assert ref.ref_io_wind(f.encode(), ga, _dp(want), len(want)) == len(ours)
    np.testing.assert_array_equal(ours, want)


@pytest.mark.parametrize("seed", [0, 1])
def test_wave_parameter_tables(ref, tmp_path, seed):
    rng = np.random.default_rng(seed)
    for jonswap, kind, ncol in ((0, inputs.XBG_TAB_WAVECST, 5), (1, inputs.XBG_TAB_JONSWAP, 6)):
        f = str(tmp_path / f"wave{jonswap}.txt")
        _table_file(f, rng, ncol, comments=False)
        ga, rt = 0.1 * seed, 1800.0
        ours = inputs.read_table(f, kind, ga, rt)
        want = np.empty_like(ours)
        assert ref.ref_io_wave(f.encode(), jonswap, ga, rt, _dp(want), len(want)) == len(ours)
        np.testing.assert_array_equal(ours, want)
    assert ours[-1, 0] == ours[-2, 0] + 1800.0       # the JONSWAP closing record


def test_bathymetry_md_and_dep(ref, tmp_path):
    rng = np.random.default_rng(4)
    nx, ny = 37, 23
    zb = rng.normal(0, 5, (ny, nx))
    f = str(tmp_path / "bathy.md")
    rows = [f"{nx}\t{ny}\t2.5\t0\t12.5"]
    order = rng.permutation(ny)                      # rows carry their own 1-based index
    for j in order:
        rows.append(f"{j + 1}\t" + "\t".join(_num(rng) if rng.random() < 0.1 else f"{v:.7g}" for v in zb[j]))
    open(f, "w").write("\n".join(rows) + "\n")
    nx2, ny2, dx, ga, ours = inputs.read_md(f)
    rnx, rny, rdx, rga = C.c_int(), C.c_int(), C.c_double(), C.c_double()
    ref.ref_io_md_head(f.encode(), C.byref(rnx), C.byref(rny), C.byref(rdx), C.byref(rga))
    assert (nx2, ny2, dx) == (rnx.value, rny.value, rdx.value) == (nx, ny, 2.5)
    assert ga == rga.value * math.pi / 180.0
    want = np.empty((ny, nx), np.float32)
    ref.ref_io_md(f.encode(), want.ctypes.data_as(C.POINTER(C.c_float)))
    np.testing.assert_array_equal(ours, want)
    f = str(tmp_path / "bathy.dep")
    with open(f, "w") as fh:
        for j in range(ny):
            fh.write("  ".join(f"{v:.6e}" for v in zb[j]) + "\n")
    ours = inputs.read_dep(f, nx, ny)
    want = np.empty((ny, nx), np.float32)
    ref.ref_io_dep(f.encode(), nx, ny, want.ctypes.data_as(C.POINTER(C.c_float)))
    np.testing.assert_array_equal(ours, want)


def test_xbeach_reuse_boundary(ref, tmp_path, monkeypatch):
    rng = np.random.default_rng(5)
    monkeypatch.chdir(tmp_path)                      # entry file names resolve here, as in the reference
    ny, nt, dtbc, rt = 9, 6, 0.5, 10.0
    nrec = math.ceil(rt / dtbc)
    lines = ["-45 45 15 0.5 10"]
    for k in range(3):
        q = rng.normal(size=4 * ny * nrec)
        E = rng.random(nt * ny * nrec) * 100
        q.astype("<f8").tofile(f"q{k}.bin")
        E.astype("<f8").tofile(f"E{k}.bin")
        lines.append(f"{k * rt}\t{8 + k * 0.37}\tq{k}.bin\tE{k}.bin")
    open("list.txt", "w").write("\n".join(lines) + "\n")
    xb = inputs.XBeachReuse("list.txt")
    hdr = np.empty(5)
    ref.ref_io_xbhead(b"list.txt", _dp(hdr))
    assert [xb.thetamin, xb.thetamax, xb.dtheta, xb.dtbc, xb.rtlength] == list(hdr)
    t, tr = np.empty(8), np.empty(8)
    n = ref.ref_io_xblist(b"list.txt", rt, _dp(t), _dp(tr), 8)
    np.testing.assert_array_equal(xb.time, t[:n])
    np.testing.assert_array_equal(xb.Trep, tr[:n])
    for k in range(3):
        St, q, trep = xb.step(k, ny, nt)
        qw, Sw, trw = np.empty(4 * ny * nrec), np.empty(nt * ny * nrec), C.c_double()
        ref.ref_io_xbstep(b"list.txt", rt, dtbc, 17, ny, nt, k, _dp(qw), _dp(Sw), C.byref(trw))
        np.testing.assert_array_equal(q.ravel(), qw)
        np.testing.assert_array_equal(St.ravel(), Sw)
        assert trep == trw.value


@pytest.mark.parametrize("sep", ["\t", " ", ","])
def test_swan_spectrum_list(ref, tmp_path, sep):
    """ReadSPECBnd's list (time, spectrum file) with each separator, blank
    lines, and the closing record, as the reference reads it."""
    rng = np.random.default_rng(len(sep))
    lines = []
    for k in range(7):
        lines.append(f"{k * 1800.0 + rng.uniform(0, 5):.6g}{sep}spec_{k:03d}_{rng.integers(1000)}.sp2")
        if k == 3:
            lines.append("")
    f = tmp_path / "specs.txt"
    f.write_text("\n".join(lines) + "\n")
    t, names = inputs.read_spec_list(f, 3600.0)
    wt = np.empty(16)
    wn = C.create_string_buffer(16 * 256)
    n = ref.ref_io_speclist(str(f).encode(), 3600.0, _dp(wt), wn, 256, 16)
    assert n == len(t) == 8
    np.testing.assert_array_equal(t, wt[:n])
    assert names == [wn.raw[k * 256:(k + 1) * 256].split(b"\0", 1)[0].decode() for k in range(n)]
    assert names[-1] == names[-2] and t[-1] == t[-2] + 3600.0


def test_malformed_files(tmp_path):
    from xbeach_gpu_b200.model import XbgError
    f = tmp_path / "bad.txt"
    f.write_text("0.0\t1.0\n5.0\n")                  # a line with one value
    with pytest.raises(XbgError, match="format"):
        inputs.read_sealevel(f)
    f.write_text("0.0 abc 1.0\n")
    with pytest.raises(XbgError, match="format"):
        inputs.read_wind(f)
    with pytest.raises(XbgError, match="opened"):
        inputs.read_sealevel(tmp_path / "missing.txt")
    f.write_text("0.0\n")                          # a spectrum list line without its file
    with pytest.raises(XbgError, match="format"):
        inputs.read_spec_list(f, 3600.0)
    f.write_text("3\t2\t1.0\t0\t0\n1 1 2 3\n2 1 2\n")   # short last row
    with pytest.raises(XbgError, match="format"):
        inputs.read_md(f)
