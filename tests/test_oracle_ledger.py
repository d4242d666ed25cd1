"""The sediment ledger of the CUDA step (test_mass.py) is a property of the
reference algorithm: the oracle's Conc + bedupdate (Sediment_kernel.cu:721-780,
881-968) close the same interior ledger, on the CPU."""
import pytest

import pyoracle
from test_mass import _sed_case, _sed_start, sediment_ledger
from xbeach_gpu_b200.abi import XBG_FP32, XBG_FP64


@pytest.mark.parametrize("precision,tol", [(XBG_FP64, 1e-12), (XBG_FP32, 1e-6)])
def test_oracle_sediment_ledger_closes(precision, tol):
    p, zb, bnd = _sed_case()
    o = pyoracle.Oracle(p, precision)
    _sed_start(o, p, zb, bnd)
    sediment_ledger(o, p, tol, steps=2)
