"""Shared set-up for the parity tests: seeded random states on small grids,
the same inputs applied to any handle (CUDA Model, Oracle, RefEmu), and the
field comparison used by every parity check."""
import numpy as np

from xbeach_gpu_b200.scenarios import make_case, random_state

WAVE_OUT = ["ee", "rr", "k", "c", "cg", "E", "H", "D", "R", "DR", "thetamean", "Fx", "Fy", "urms", "ust"]
FLOWBND_OUT = ["uu", "zs", "vv", "umeanbnd"]
FLOW_OUT = ["uu", "vv", "zs", "hh", "hu", "hv", "hum", "hvm", "qx", "qy", "dzsdt", "ueu", "vev",
            "vmageu", "vmagev", "vu", "uv", "uuold", "vvold", "zsold", "wetu", "wetv"]
SED_OUT = ["C", "ceqsg", "zb", "hh", "zs", "stdep", "dzb", "cfm", "fwm", "rolthick", "kturb"]
MEANS_OUT = ["Hmean", "uumean", "vvmean", "hhmean", "zsmean", "Cmean", "zsmax"]


def small_params(nx=40, ny=24, ntheta=6, **kw):
    p, zb, bnd = make_case("linear_beach", nx=nx, ny=ny, ntheta=ntheta)
    for k, v in kw.items():
        setattr(p, k, v)
    return p, bnd


def random_inputs(p, seed, steep=False):
    f = random_state(p, seed=seed)
    rng = np.random.default_rng(seed + 1000)
    if steep:   # bed slopes beyond wetdzmax/drydzmax so that avalanching acts
        f["zb"] = f["zb"] + rng.normal(0, 1.5, f["zb"].shape) * p.dx * 0.2
        f["hh"] = np.maximum(f["zb"] + f["zs"], p.eps)
    wet = (rng.random(p.nx * p.ny) > 0.1).astype(np.int32)
    f["wetu"] = wet
    f["wetv"] = np.roll(wet, 3)
    return f


def apply(h, f):
    for k, v in f.items():
        h.set(k, v)


def rel_err(a, b, floor=1e-12):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    scale = max(np.abs(b).max(), floor)
    return float(np.abs(a - b).max() / scale)


def compare(h1, h2, names, tol, what=""):
    bad = []
    for n in names:
        e = rel_err(h1.get(n), h2.get(n))
        if not (e <= tol):
            bad.append((n, e))
    assert not bad, f"{what}: fields above {tol:g} relative error: {bad}"
