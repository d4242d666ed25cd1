"""Generate the golden fixtures of tests/golden/ from the reference itself.

Runs the reference's own CPU wave code (wave_CPU.cpp) and its own flow and
sediment CUDA kernels (run on the CPU, oracle/_ref/libxbg_ref.so, built in
place from the reference checkout by oracle/Makefile) on seeded small cases
and stores inputs and outputs of each phase.  Regenerate with

    python tests/golden/make_golden.py

(needs the reference checkout; the fixtures themselves are committed).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")]

import pyoracle  # noqa: E402
from helpers import (FLOW_OUT, FLOWBND_OUT, SED_OUT, WAVE_OUT, random_inputs,  # noqa: E402
                     small_params)

CASES = {
    "roelvink_roller": dict(nx=24, ny=16, ntheta=6, seed=11, steep=False, kw={}),
    "baldock_wci_odd": dict(nx=23, ny=13, ntheta=9, seed=12, steep=False,
                            kw=dict(breakmodel=2, wci=0.6)),
    "steep_noroller": dict(nx=24, ny=16, ntheta=4, seed=13, steep=True,
                           kw=dict(roller=0, morfac=10.0)),
}
STEP = dict(dt=0.31, t=37.3)


def step_inputs(p, bnd):
    """The host-side boundary values of one step, computed as wavebnd/flowbnd
    do (Wavestep.cu:684-741, Wave_gpu.cu:1020-1073) for record 37..38."""
    t = STEP["t"]
    nb = int(np.floor(t / p.dtbc))
    tn, ts = p.dtbc, t - nb * p.dtbc
    so = bnd["St"][nb].astype(np.float32).astype(np.float64)
    sn = bnd["St"][nb + 1].astype(np.float32).astype(np.float64)
    St = (so + ts / tn * (sn - so)).astype(np.float32)
    qo = bnd["q"][nb].astype(np.float32)
    qn = bnd["q"][nb + 1].astype(np.float32)
    return dict(St=St, qold=qo, qnew=qn, timesincelast=ts, timenext=tn, zsbndi=0.12, zsbndn=0.31,
                windu=4.0, windv=-1.5)


def run_case(name, c):
    p, bnd = small_params(c["nx"], c["ny"], c["ntheta"], **c["kw"])
    f = random_inputs(p, c["seed"], steep=c["steep"])
    r = pyoracle.RefEmu(p)
    for k, v in f.items():
        r.set(k, v)
    si = step_inputs(p, bnd)
    r.step_inputs(STEP["dt"], STEP["t"], np.float32(bnd["Trep"]), si["St"], si["qold"], si["qnew"],
                  si["timesincelast"], si["timenext"], si["zsbndi"], si["zsbndn"], si["windu"], si["windv"])
    out = {"in_" + k: np.asarray(r.get(k)) for k in f}
    r.call("wave_step")
    out.update({"wave_" + k: r.get(k) for k in WAVE_OUT})
    r.call("flow_boundary")
    out.update({"fbnd_" + k: r.get(k) for k in FLOWBND_OUT})
    r.call("flow_step")
    out.update({"flow_" + k: r.get(k) for k in FLOW_OUT})
    r.call("sediment_step")
    out.update({"sed_" + k: r.get(k) for k in SED_OUT})
    for k, v in si.items():
        out["si_" + k] = np.asarray(v)
    out["Trep"] = np.float32(bnd["Trep"])
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
    print(name, len(out), "arrays")


if __name__ == "__main__":
    pyoracle.build(ref=True)
    for n, c in CASES.items():
        run_case(n, c)
