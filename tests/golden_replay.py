"""Replay a golden case (tests/golden/*.npz, produced from the reference
itself by tests/golden/make_golden.py) on any handle with the C-ABI call
sequence, phase by phase."""
import os

import numpy as np

from golden.make_golden import CASES, STEP
from helpers import FLOW_OUT, FLOWBND_OUT, SED_OUT, WAVE_OUT, small_params

HERE = os.path.dirname(os.path.abspath(__file__))
PHASES = [("wave", "wave_step", WAVE_OUT), ("fbnd", "flow_boundary", FLOWBND_OUT),
          ("flow", "flow_step", FLOW_OUT), ("sed", "sediment_step", SED_OUT)]


def load(name):
    return dict(np.load(os.path.join(HERE, "golden", f"{name}.npz")))


def setup(handle_cls, name, **kw):
    c = CASES[name]
    p, bnd = small_params(c["nx"], c["ny"], c["ntheta"], **c["kw"])
    g = load(name)
    h = handle_cls(p, **kw)
    h.set_wave_boundary(0, bnd["St"], bnd["q"], t0=0.0, tend=p.rtlength, Trep=bnd["Trep"])
    si = {k[3:]: g[k] for k in g if k.startswith("si_")}
    h.set_sealevel([0.0, 1e6], [float(si["zsbndi"])] * 2, [float(si["zsbndn"])] * 2)
    h.set_wind([0.0, 1e6], [float(si["windu"])] * 2, [float(si["windv"])] * 2)
    for k in g:
        if k.startswith("in_"):
            h.set(k[3:], g[k])
    return p, h, g


def start_step(h, p):
    """Put the handle at the golden step's time and dt, as the reference host
    code had computed them, and run the boundary interpolation."""
    h.set_time(STEP["t"], STEP["dt"], STEP["dt"])
