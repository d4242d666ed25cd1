"""Seeded synthetic cases with the shapes of the reference's workloads.

There is no public dataset for this path: every case is generated here.  The
conventions are the reference's: zb is bed depth positive down, hh = zb + zs
(Wave_gpu.cu:2009-2010), the offshore boundary is column ix = 0, angles in
radians, directional boundary energy St[record][itheta][iy] (Stfile layout,
Wavestep.cu:703-706) and bound-long-wave fluxes q[record][4][iy] (qfile
layout, Wavestep.cu:709-712).

Cases
  linear_beach   nx=200 ny=100 dx=5 m, 1:50 slope from 10 m depth to +2 m
                 land, 10 directional bins of 10 deg over -50..50 deg,
                 Hm0 1.5 m, Tp 10 s, D50 0.2 mm, morfac 1 (the reference's
                 CPU-runnable case).
  barred_beach   nx=2048 ny=1024 dx=2 m, 1:40 base slope capped at 15 m,
                 Gaussian bar (1.5 m, 150 m offshore of the waterline, 40 m
                 wide) whose crest varies alongshore (250 m, 0.5 m), 5 cm
                 seeded noise, 18 bins over -90..90 deg, Hm0 2.5 m, Tp 12 s,
                 D50 0.25 mm, morfac 10 (the large single domain).
  ensemble       (make_ensemble) n scenarios of uneven grids: nx uniform on
                 [128, 1024], ny on [64, 512] in multiples of 32, dx=4 m, 12
                 bins over -90..90 deg; per scenario a slope uniform on
                 [1/100, 1/20] (depth capped at 12 m offshore, land at -3 m),
                 a Gaussian bar with probability 0.5, Hm0 on [0.5, 4] m, Tp on
                 [6, 14] s, mean direction on [-30, 30] deg, D50 on
                 [0.15, 0.4] mm, 1800 s, boundary seed = seed + k.
  storm          (iter_storm_ensemble) the surrogate-assisted ensemble: n
                 scenarios drawn as the ensemble's with nx on [256, 1024] and
                 ny on [128, 512], morfac 10, each under a 6 h storm whose Hm0
                 ramps linearly 1 -> 5 -> 1 m and Tp 8 -> 14 -> 8 s; model
                 time 0 is storm time t_start, and the boundary chunk covers
                 the next rtlength seconds.
The wave boundary is a seeded wave-group series on the bins: a cos^2s
directional spreading of the JONSWAP energy Hm0^2 rho g / 16 (as GenCstWave,
makjonswap.cpp:24-70, spreads it) modulated in time by a sum of random-phase
group components, with a matching bound-long-wave flux.  It stands in for
GenWGnLBW's output (makjonswap.cpp:235) with the same array shapes.
"""
import math

import numpy as np

from .abi import default_params, sanity

PI = 3.14159265


def wave_group_boundary(p, nrec, Hs, Tp, mean_dir, s=10.0, seed=0, ngroup=8, dtbc=1.0):
    """St[nrec][ntheta][ny] and q[nrec][4][ny] (float64) for the bins of p."""
    rng = np.random.default_rng(seed)
    nt, ny = p.ntheta, p.ny
    theta = np.array([i * p.dtheta + p.thetamin + 0.5 * p.dtheta for i in range(nt)], dtype=np.float32)
    eetot = Hs * Hs * p.rho * p.g / (16.0 * p.dtheta)
    scaled = np.cos((theta.astype(np.float64) - mean_dir) / 2.0) ** (2.0 * s)
    Stdir = scaled / scaled.sum() * eetot
    t = np.arange(nrec) * dtbc
    yy = np.arange(ny) * p.dx
    fgroup = rng.uniform(0.5, 1.5, ngroup) / (8.0 * Tp)
    ky = rng.uniform(-1.0, 1.0, ngroup) * 2 * math.pi / max(ny * p.dx, 1.0)
    ph = rng.uniform(0, 2 * math.pi, ngroup)
    env = np.zeros((nrec, ny))
    for f, k, a in zip(fgroup, ky, ph):
        env += np.cos(2 * math.pi * f * t[:, None] + k * yy[None, :] + a)
    env = 1.0 + 0.6 * env / math.sqrt(ngroup)
    env = np.clip(env, 0.05, None)
    St = env[:, None, :] * Stdir[None, :, None]
    q = np.zeros((nrec, 4, ny))
    q[:, 0, :] = 0.02 * Hs * (env - env.mean())
    q[:, 1, :] = 0.005 * Hs * (env - env.mean())
    return St, q


def make_case(name, seed=0, nx=None, ny=None, ntheta=None):
    """Return (params, zb[ny,nx] float64, boundary dict) for a named case."""
    p = default_params()
    rng = np.random.default_rng(seed)
    if name == "linear_beach":
        p.nx, p.ny, p.dx = nx or 200, ny or 100, 5.0
        p.thetamin, p.thetamax = -50 * PI / 180, 50 * PI / 180
        p.dtheta = 10 * PI / 180
        if ntheta:
            p.dtheta = (p.thetamax - p.thetamin) / ntheta
        x = np.arange(p.nx) * p.dx
        zb = np.maximum(10.0 - x / 50.0, -2.0)[None, :].repeat(p.ny, axis=0)
        Hs, Tp, mdir = 1.5, 10.0, 0.0
        p.D50, p.D90, p.morfac, p.endtime = 0.0002, 0.0003, 1.0, 600.0
    elif name == "barred_beach":
        p.nx, p.ny, p.dx = nx or 2048, ny or 1024, 2.0
        p.thetamin, p.thetamax = -90 * PI / 180, 90 * PI / 180
        p.dtheta = 10 * PI / 180
        if ntheta:
            p.dtheta = (p.thetamax - p.thetamin) / ntheta
        x = np.arange(p.nx) * p.dx
        y = np.arange(p.ny) * p.dx
        xw = 0.83 * p.nx * p.dx
        base = np.clip((xw - x) / 40.0, -3.0, 15.0)
        bar = 1.5 * (1 + (0.5 / 1.5) * np.sin(2 * math.pi * y / 250.0))[:, None] * \
            np.exp(-(((x - (xw - 150.0)) / 40.0) ** 2) / 2)[None, :]
        zb = base[None, :] - bar + rng.normal(0.0, 0.05, (p.ny, p.nx))
        Hs, Tp, mdir = 2.5, 12.0, 10 * PI / 180
        p.D50, p.D90, p.morfac, p.endtime = 0.00025, 0.000375, 10.0, 3600.0
    else:
        raise ValueError(name)
    p.wavebndtype = 4
    p.sedtrans, p.morphology, p.sedstart = 1, 1, 0.0
    p.CFL, p.eps = 0.7, 0.01
    p.dtbc, p.rtlength = 1.0, 3600.0
    p = sanity(p, endbnd=1e9)
    nrec = int(math.ceil(p.rtlength / p.dtbc)) + 1
    St, q = wave_group_boundary(p, nrec, Hs, Tp, mdir, seed=seed + 1)
    bnd = dict(St=St, q=q, t0=0.0, tend=p.rtlength, Trep=Tp / 1.1, Hs=Hs, Tp=Tp)
    return p, zb, bnd


def random_state(p, seed=0, wet_fraction=0.85):
    """Physically plausible random fields for per-kernel tests on small grids."""
    rng = np.random.default_rng(seed)
    nx, ny, nt = p.nx, p.ny, p.ntheta
    x = np.arange(nx)
    zb = (6.0 - 8.0 * x / nx)[None, :] + rng.normal(0, 0.3, (ny, nx))
    zs = 0.1 * rng.standard_normal((ny, nx))
    zs = np.maximum(zs, -zb)
    hh = np.maximum(zb + zs, p.eps)
    f = {}
    f["zb"], f["zs"], f["hh"] = zb, zs, hh
    f["uu"] = 0.5 * rng.standard_normal((ny, nx))
    f["vv"] = 0.3 * rng.standard_normal((ny, nx))
    f["hu"] = np.maximum(hh + 0.05 * rng.standard_normal((ny, nx)), 0)
    f["hv"] = np.maximum(hh + 0.05 * rng.standard_normal((ny, nx)), 0)
    f["hum"], f["hvm"] = hh.copy(), hh.copy()
    f["qx"] = f["uu"] * f["hu"]
    f["qy"] = f["vv"] * f["hv"]
    f["uuold"] = f["uu"] + 0.05 * rng.standard_normal((ny, nx))
    f["vvold"] = f["vv"] + 0.05 * rng.standard_normal((ny, nx))
    f["zsold"] = zs + 0.02 * rng.standard_normal((ny, nx))
    f["ueu"], f["vev"] = f["uu"] * 0.9, f["vv"] * 0.9
    f["vmageu"] = np.hypot(f["ueu"], f["vv"])
    f["vmagev"] = np.hypot(f["uu"], f["vev"])
    f["vu"], f["uv"] = f["vv"] * 0.8, f["uu"] * 0.8
    f["H"] = np.abs(0.8 + 0.3 * rng.standard_normal((ny, nx)))
    f["E"] = p.rho * p.g * f["H"] ** 2 / 8
    f["DR"] = np.abs(50 * rng.standard_normal((ny, nx)))
    f["R"] = np.abs(100 * rng.standard_normal((ny, nx)))
    f["D"] = np.abs(50 * rng.standard_normal((ny, nx)))
    f["c"] = np.sqrt(p.g * hh) + 0.5
    f["cg"] = f["c"] * 0.9
    f["k"] = 2 * math.pi / (f["c"] * 10.0)
    f["Fx"] = 5 * rng.standard_normal((ny, nx))
    f["Fy"] = 2 * rng.standard_normal((ny, nx))
    f["urms"] = np.abs(0.4 * rng.standard_normal((ny, nx)))
    f["ust"] = np.abs(0.1 * rng.standard_normal((ny, nx)))
    f["thetamean"] = 0.3 * rng.standard_normal((ny, nx))
    f["cfm"] = np.full((ny, nx), 0.01)
    f["fwm"] = np.full((ny, nx), 0.001)
    f["C"] = np.abs(1e-4 * rng.standard_normal((ny, nx)))
    f["stdep"] = np.abs(5 + rng.standard_normal((ny, nx)))
    f["dzsdt"] = 1e-3 * rng.standard_normal((ny, nx))
    f["rolthick"] = np.abs(0.1 * rng.standard_normal((ny, nx)))
    f["umeanbnd"] = 0.01 * rng.standard_normal(ny)
    ee = np.abs(200 * rng.standard_normal((nt, ny, nx)) + 300)
    ee *= (rng.random((nt, ny, nx)) > 0.1)
    rr = np.abs(50 * rng.standard_normal((nt, ny, nx)))
    f["ee"], f["rr"] = ee, rr
    dry = rng.random((ny, nx)) > wet_fraction
    f["hh"] = np.where(dry, p.eps, f["hh"])
    return f


def make_ensemble(n, seed=0, **kw):
    """n scenarios of the ragged ensemble: a list of (params, zb, boundary)."""
    return list(iter_ensemble(n, seed, **kw))


def iter_ensemble(n, seed=0, nx_range=(128, 1024), ny_range=(64, 512), step=32, dx=4.0, ntheta=12,
                  endtime=1800.0, dtbc=5.0, boundary=True):
    """The scenarios of make_ensemble one at a time.  The boundary records are
    dtbc apart (the groups' time scales are tens of seconds), which keeps a
    scenario's chunk a few MB.  boundary=False yields the parameters and bed
    only (boundary None) with the same random draws."""
    rng = np.random.default_rng(seed)
    for k in range(n):
        p = default_params()
        p.nx = int(rng.integers(nx_range[0] // step, nx_range[1] // step + 1)) * step
        p.ny = int(rng.integers(ny_range[0] // step, ny_range[1] // step + 1)) * step
        p.dx = dx
        p.thetamin, p.thetamax = -90 * PI / 180, 90 * PI / 180
        p.dtheta = (p.thetamax - p.thetamin) / ntheta
        slope = rng.uniform(1 / 100, 1 / 20)
        x = np.arange(p.nx) * p.dx
        y = np.arange(p.ny) * p.dx
        xw = 0.8 * p.nx * p.dx
        zb = np.clip((xw - x) * slope, -3.0, 12.0)[None, :].repeat(p.ny, axis=0)
        if rng.random() < 0.5:
            xb = xw - rng.uniform(0.1, 0.3) * xw
            zb = zb - 1.5 * np.exp(-(((x - xb) / 40.0) ** 2) / 2)[None, :]
        Hs, Tp = rng.uniform(0.5, 4.0), rng.uniform(6.0, 14.0)
        mdir = rng.uniform(-30.0, 30.0) * PI / 180
        p.D50 = rng.uniform(0.00015, 0.0004)
        p.D90 = 1.5 * p.D50
        p.morfac, p.endtime = 1.0, endtime
        p.wavebndtype = 4
        p.sedtrans, p.morphology, p.sedstart = 1, 1, 0.0
        p.CFL, p.eps = 0.7, 0.01
        p.dtbc, p.rtlength = dtbc, endtime
        p = sanity(p, endbnd=1e9)
        nrec = int(math.ceil(p.rtlength / p.dtbc)) + 1
        if not boundary:
            yield p, zb, None
            continue
        St, q = wave_group_boundary(p, nrec, Hs, Tp, mdir, seed=seed + 1 + k, dtbc=dtbc)
        bnd = dict(St=St, q=q, t0=0.0, tend=p.rtlength, Trep=Tp / 1.1, Hs=Hs, Tp=Tp)
        yield p, zb, bnd


STORM_S = 6 * 3600.0


def storm_hs_tp(tau):
    """Hm0 and Tp of the 6 h storm at storm time tau [s]: linear 1 -> 5 -> 1 m
    and 8 -> 14 -> 8 s, peaking at 3 h."""
    r = 1.0 - abs(2.0 * np.clip(tau, 0.0, STORM_S) / STORM_S - 1.0)
    return 1.0 + 4.0 * r, 8.0 + 6.0 * r


def iter_storm_ensemble(n, seed=0, nx_range=(256, 1024), ny_range=(128, 512), step=32, dx=4.0, ntheta=12,
                        t_start=7200.0, rtlength=3600.0, dtbc=5.0, boundary=True, t_start_range=None):
    """The storm scenarios one at a time: (params, zb, boundary) as
    iter_ensemble gives them, morfac 10, with the boundary chunk of storm
    times [t_start, t_start + rtlength): St scaled per record by Hm0(t)^2
    (the wave energy) and q by Hm0(t) from a unit-height group series, Trep
    from Tp at the chunk's middle; boundary["storm"] maps model time to
    (Hm0, Tp).  t_start_range = (a, b): each scenario starts at its own
    storm time drawn uniformly from [a, b] (training sets that span the
    storm)."""
    base = iter_ensemble(n, seed, nx_range=nx_range, ny_range=ny_range, step=step, dx=dx, ntheta=ntheta,
                         endtime=rtlength, dtbc=dtbc, boundary=False)
    rng = np.random.default_rng(seed + 7777)
    for k, (p, zb, _) in enumerate(base):
        p.morfac = 10.0
        mdir = rng.uniform(-30.0, 30.0) * PI / 180
        ts = t_start if t_start_range is None else float(rng.uniform(*t_start_range))
        if not boundary:
            yield p, zb, None
            continue
        nrec = int(math.ceil(p.rtlength / p.dtbc)) + 1
        hs_mid, tp_mid = storm_hs_tp(ts + 0.5 * rtlength)
        St, q = wave_group_boundary(p, nrec, 1.0, tp_mid, mdir, seed=seed + 1 + k, dtbc=p.dtbc)
        hs_t = storm_hs_tp(ts + np.arange(nrec) * p.dtbc)[0]
        St = St * (hs_t ** 2)[:, None, None]
        q = q * hs_t[:, None, None]
        bnd = dict(St=St, q=q, t0=0.0, tend=p.rtlength, Trep=tp_mid / 1.1, Hs=hs_mid, Tp=tp_mid,
                   storm=lambda t, t0=ts: storm_hs_tp(t0 + t))
        yield p, zb, bnd
