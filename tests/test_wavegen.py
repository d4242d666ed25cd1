"""The offshore boundary generators (include/xbg_bnd.h) against the
reference's own (makjonswap.cpp: makjonswap + GenWGnLBW, GenCstWave),
compiled in place into oracle/_ref/libxbg_ref_wavegen.so with an exact-DFT
stand-in for FFTW (FFTW is not installed; it computes the same transforms to
rounding, so this pins the arithmetic, not FFTW's own rounding).

Wave groups: the library's random phases and directions are the reference's
draws (same engine and order), the transforms are sums in double on the
GPU, the envelope a radix-2 FFT; St and q agree with the reference's to
1e-9 of their largest magnitude and Trep exactly.  Constant waves: host
arithmetic in the reference's order, bit for bit."""
import ctypes as C
import math
import os
import re

import numpy as np
import pytest

from xbeach_gpu_b200 import boundary
from xbeach_gpu_b200.abi import default_params

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_WG = os.path.join(ROOT, "oracle", "_ref", "libxbg_ref_wavegen.so")
TOL = 1e-9


@pytest.fixture(scope="module")
def ref():
    if not os.path.exists(REF_WG):
        pytest.skip("oracle/_ref/libxbg_ref_wavegen.so not built (needs the reference checkout)")
    L = C.CDLL(REF_WG)
    vp = C.c_void_p
    L.ref_wavegen.argtypes = [vp, vp, vp, vp, vp, vp]
    L.ref_gencst.argtypes = [vp, vp, vp, C.c_int, vp, vp, vp, vp]
    return L


def _params(ny, ntheta, thetamin_deg, dtheta_deg, rtlength, dtbc=1.0, dx=5.0):
    p = default_params()
    p.ny, p.nx, p.dx = ny, 16, dx
    p.ntheta = ntheta
    p.thetamin, p.dtheta = math.radians(thetamin_deg), math.radians(dtheta_deg)
    p.thetamax = p.thetamin + ntheta * p.dtheta
    p.dtbc, p.rtlength = dtbc, rtlength
    return p


def _ref_groups(L, p, w):
    pi_ = np.array([p.ny, p.ntheta, 0, w.nspr], np.int32)
    pd = np.array([p.dx, p.thetamin, p.dtheta, p.dtbc, p.rtlength, p.rho, p.g, w.sprdthr, w.offdepth, w.nmax,
                   w.fcutoff], np.float64)
    ww = np.array([w.Hs, w.Tp, w.Dp, w.s, w.gamma], np.float64)
    nrec = int(math.ceil(p.rtlength / p.dtbc)) + 1
    St = np.zeros(nrec * p.ntheta * p.ny)
    q = np.zeros(nrec * 4 * p.ny)
    tr = np.zeros(1)
    L.ref_wavegen(pi_.ctypes.data, pd.ctypes.data, ww.ctypes.data, St.ctypes.data, q.ctypes.data, tr.ctypes.data)
    return St.reshape(nrec, p.ntheta, p.ny), q.reshape(nrec, 4, p.ny), tr[0]


def _err(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


CASES = {
    "normal": (dict(ny=12, ntheta=6, thetamin_deg=-45, dtheta_deg=15, rtlength=200.0),
               dict(Hs=1.5, Tp=10.0, Dp=0.0, s=10.0, gamma=3.3, offdepth=10.0)),
    "oblique_nspr_cutoff": (dict(ny=9, ntheta=8, thetamin_deg=-60, dtheta_deg=15, rtlength=240.0, dx=8.0),
                            dict(Hs=2.5, Tp=12.0, Dp=math.radians(20.0), s=20.0, gamma=2.0, offdepth=15.0,
                                 nspr=1, fcutoff=0.01)),
    "short_steep": (dict(ny=7, ntheta=5, thetamin_deg=-50, dtheta_deg=20, rtlength=150.0, dtbc=0.5),
                    dict(Hs=1.0, Tp=6.0, Dp=math.radians(-10.0), s=5.0, gamma=5.0, offdepth=6.0)),
}


@pytest.mark.gpu
@pytest.mark.parametrize("case", sorted(CASES))
def test_wave_groups_match_reference(ref, case):
    pk, wk = CASES[case]
    p = _params(**pk)
    w = boundary.wavegen(**wk)
    St, q, tr = boundary.wave_groups(p, w)
    Sr, qr, trr = _ref_groups(ref, p, w)
    assert tr == trr
    assert np.isfinite(St).all() and np.isfinite(q).all()
    assert St.max() > 0 and np.abs(q[:, :2]).max() > 0
    e_st, e_q = _err(St, Sr), _err(q, qr)
    assert e_st <= TOL and e_q <= TOL, (e_st, e_q)
    assert np.all(q[:, 2:] == 0.0)


def test_constant_waves_match_reference(ref):
    p = _params(ny=11, ntheta=7, thetamin_deg=-70, dtheta_deg=20, rtlength=100.0)
    theta = np.array([np.float32(p.thetamin + (t + 0.5) * p.dtheta) for t in range(p.ntheta)], np.float32)
    rec = np.array([[0.0, 1.2, 9.0, 0.1, 10.0], [50.0, 2.0, 11.0, -0.3, 4.0], [80.0, 0.7, 7.5, 0.0, 25.0]])
    St, q, Tp = boundary.constant_waves(p, rec, theta.astype(np.float64))
    n = rec.shape[0]
    Sr, qr, Tr = np.zeros(n * p.ntheta * p.ny), np.zeros(n * 4 * p.ny), np.zeros(n)
    pi_ = np.array([p.ny, p.ntheta, 0, 0], np.int32)
    pd = np.array([p.dx, p.thetamin, p.dtheta, p.dtbc, p.rtlength, p.rho, p.g, 0, 0, 0, 0], np.float64)
    ref.ref_gencst(pi_.ctypes.data, pd.ctypes.data, rec.ctypes.data, n, theta.ctypes.data, Sr.ctypes.data,
                   qr.ctypes.data, Tr.ctypes.data)
    np.testing.assert_array_equal(St.ravel(), Sr)
    np.testing.assert_array_equal(q.ravel(), qr)
    np.testing.assert_array_equal(Tp, Tr)


def test_bnd_header_symbols_exported():
    from xbeach_gpu_b200 import build
    build.build(verbose=False)
    L = boundary._lib()
    txt = open(os.path.join(ROOT, "include", "xbg_bnd.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    syms = sorted(set(re.findall(r"\b(xbg_[a-z0-9_]+)\s*\(", txt)))
    assert syms == ["xbg_gen_constant_waves", "xbg_gen_wave_groups", "xbg_wavegen_default"]
    assert all(hasattr(L, s) for s in syms)


def test_refuses_bad_sizes():
    from xbeach_gpu_b200.model import XbgError
    p = _params(ny=4, ntheta=4, thetamin_deg=-40, dtheta_deg=20, rtlength=100.0)
    w = boundary.wavegen(offdepth=-1.0)
    with pytest.raises(XbgError):
        boundary.wave_groups(p, w)
