"""The C-ABI library loads on a CPU-only machine and exports every entry point
that include/xbg.h declares; the host-side parameter functions agree with
their Python twins (no GPU call is made here)."""
import ctypes as C
import os
import re

import pytest

from xbeach_gpu_b200 import abi, model

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    txt = open(os.path.join(ROOT, "include", "xbg.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(xbg_[a-z0-9_]+)\s*\(", txt)))


@pytest.fixture(scope="module")
def lib():
    from xbeach_gpu_b200 import build
    build.build(verbose=False)
    return model.load()


def test_exports_every_declared_symbol(lib):
    syms = header_symbols()
    assert len(syms) >= 25
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing
    assert sorted(model.EXPORTS) == syms


def test_params_default_matches_python(lib):
    p = abi.Params()
    lib.xbg_params_default(C.byref(p))
    q = abi.default_params()
    for k, _ in abi.Params._fields_:
        assert getattr(p, k) == pytest.approx(getattr(q, k)), k


def test_params_sanity_matches_python(lib):
    p = abi.default_params()
    p.nx, p.ny, p.dx = 64, 32, 4.0
    p.thetamin, p.thetamax, p.dtheta = -0.8, 0.8, 0.2
    q = abi.Params.from_buffer_copy(p)
    assert lib.xbg_params_sanity(C.byref(p), 900.0) == 0
    abi.sanity(q, 900.0)
    for k, _ in abi.Params._fields_:
        assert getattr(p, k) == pytest.approx(getattr(q, k)), k
    assert p.ntheta == 8 and p.endtime == 900.0 and p.nuh == p.smag and p.cfsand == p.cf


def test_status_strings(lib):
    for s in range(11):
        assert lib.xbg_status_string(s)
