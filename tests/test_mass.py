"""Water and sediment mass balances of the CUDA step.

Water.

Continuity (Flow_kernel.cu:1626-1681) and the second-order water-level
correction (wrkzs2Ocorr / zs2Ocorr, :2130-2317, which also adds its fluxes to
qx and qy) are together a flux-form update: for every cell with ix >= 1 and
1 <= iy <= ny-2,
    zs_new - zs_old = dt/dx (QX[ix-1] - QX[ix] + QY[iy-1] - QY[iy])
with the step's final fluxes QX, QY.  Summed over those cells the volume
change is the flux through the domain's faces; the lateral rows (latbnd) and
the offshore column (ubnd1D) are copies, i.e. sources by the reference's
design, and are reported separately.  The ledger closes to 1e-12 of the water
volume in FP64 and to 1e-6 in FP32.

Sediment.  Conc (Sediment_kernel.cu:721-780) solves
    cs = h C_old - dt div(Sus, Svs) + dt (ero - depo),   depo = cs / Ts,
for the new suspended load cs = C_new h, and bedupdate (:881-968) moves the
bed by dzg = morfac dt / (1 - por) (ero - depo), stored as dzb = -dzg.  So in
every interior cell (ix >= 1, 1 <= iy <= ny-2)
    C_new h - C_old h + (1 - por) / morfac * dzb = -dt div(Sus, Svs),
and over the interior the divergence telescopes to the fluxes through the
interior's outer faces.  With no suspended sediment within three cells of the
domain edge those fluxes are zero, so the suspended plus bed sediment of the
interior is conserved; the lateral copies (CClatbnd, zblatbnd), C = 0 at
ix = 0, the clipping of cs to [0, 0.1 h] and the dry-cell zeroing are the
sources by the reference's design (none of them acts in the case below).
The ledger closes to 1e-12 in FP64 and 1e-6 in FP32."""
import numpy as np
import pytest

from xbeach_gpu_b200.abi import XBG_FP32, XBG_FP64
from xbeach_gpu_b200.model import Model
from xbeach_gpu_b200.scenarios import make_case

pytestmark = pytest.mark.gpu


def _model(precision):
    p, zb, bnd = make_case("linear_beach", nx=96, ny=48, ntheta=10)
    p.sedtrans = 0          # bed updates also move zs; this ledger is the flow's
    m = Model(p, precision)
    m.set_wave_boundary(0, bnd["St"], bnd["q"], t0=0.0, tend=p.rtlength, Trep=bnd["Trep"])
    m.set_sealevel([0.0, 1e6], [0.0, 0.0], [0.0, 0.0])
    m.set_wind([0.0, 1e6], [0.0, 0.0], [0.0, 0.0])
    m.init_state(zb, 0.0, 0.0)
    m.advance(120)          # waves and set-up develop, the shoreline moves
    return p, m


@pytest.mark.parametrize("precision,tol", [(XBG_FP64, 1e-12), (XBG_FP32, 1e-6)])
def test_water_ledger_closes(precision, tol):
    p, m = _model(precision)
    nx, ny, dx = p.nx, p.ny, p.dx
    for _ in range(5):
        m.compute_dt()
        m.wave_boundary()
        m.flow_boundary()
        zs0 = m.get("zs").reshape(ny, nx).astype(np.float64)
        m.wave_step()
        m.flow_step()
        m.accumulate_means()
        zs1 = m.get("zs").reshape(ny, nx).astype(np.float64)
        QX = m.get("qx").reshape(ny, nx).astype(np.float64)
        QY = m.get("qy").reshape(ny, nx).astype(np.float64)
        hh = m.get("hh").reshape(ny, nx).astype(np.float64)
        dt = m.time()[1]
        # per cell, in the interior
        I = (slice(1, ny - 1), slice(1, nx))
        div = np.zeros((ny, nx))
        div[1:ny - 1, 1:] = (QX[1:ny - 1, :-1] - QX[1:ny - 1, 1:] + QY[0:ny - 2, 1:] - QY[1:ny - 1, 1:]) / dx
        dz = zs1 - zs0
        scale = np.abs(zs1).max() + np.abs(hh).max()
        assert np.abs(dz[I] - dt * div[I]).max() <= 50 * tol * scale
        # globally: interior volume change = flux through the faces
        dV = dz[I].sum() * dx * dx
        F = dt * dx * ((QX[1:ny - 1, 0] - QX[1:ny - 1, nx - 1]).sum() + (QY[0, 1:] - QY[ny - 2, 1:]).sum())
        V = hh.sum() * dx * dx
        assert abs(dV - F) <= tol * V, (dV, F, V)
        assert abs(F) > 0                      # water does cross the faces
    m.close()


def _sed_case():
    p, zb, bnd = make_case("linear_beach", nx=96, ny=48, ntheta=10)
    p.morfac = 10.0
    return p, zb, bnd


def _sed_start(h, p, zb, bnd):
    h.set_wave_boundary(0, bnd["St"], bnd["q"], t0=0.0, tend=p.rtlength, Trep=bnd["Trep"])
    h.set_sealevel([0.0, 1e6], [0.0, 0.0], [0.0, 0.0])
    h.set_wind([0.0, 1e6], [0.0, 0.0], [0.0, 0.0])
    h.init_state(zb, 0.0, 0.0)
    h.advance(120)          # waves, set-up and currents develop; the bed starts to move


def sediment_ledger(h, p, tol, steps=4):
    """Run `steps` coupled steps on handle h (CUDA Model or the oracle), each
    with a fresh sediment cloud, and check the interior sediment ledger."""
    nx, ny = p.nx, p.ny
    x = np.arange(nx)[None, :]
    y = np.arange(ny)[:, None]
    k = 1.0 - p.por
    for step in range(steps):
        for call in ("compute_dt", "wave_boundary", "flow_boundary", "wave_step", "flow_step"):
            h.call(call)
        hh = h.get("hh").reshape(ny, nx).astype(np.float64)
        # a smooth suspended-sediment cloud over the wet surf zone, zero within
        # three cells of every edge and of any dry cell
        wet = hh > 4 * p.eps
        near_dry = np.zeros_like(wet)
        for dy in range(-3, 4):
            for dx in range(-3, 4):
                near_dry |= ~np.roll(np.roll(wet, dy, 0), dx, 1)
        c0 = 2e-4 * np.exp(-((x - 0.45 * nx) / (0.2 * nx)) ** 2 - ((y - 0.5 * ny) / (0.25 * ny)) ** 2)
        c0 = np.where(near_dry, 0.0, c0)
        c0[:, :3] = 0.0; c0[:, -3:] = 0.0; c0[:3, :] = 0.0; c0[-3:, :] = 0.0
        h.set("C", c0)
        c_old = h.get("C").reshape(ny, nx).astype(np.float64)
        h.call("sediment_step")
        h.call("accumulate_means")
        c_new = h.get("C").reshape(ny, nx).astype(np.float64)
        dzb = h.get("dzb").reshape(ny, nx).astype(np.float64)
        I = (slice(1, ny - 1), slice(1, nx))
        assert wet[I].sum() > 0.5 * wet[I].size
        cs = c_new * hh
        assert not np.any((cs[I] >= 0.1 * hh[I] * (1 - 1e-6)) & wet[I])   # no clipping at 0.1 h
        bed = k / p.morfac * dzb
        susp = cs - c_old * hh
        ledger = (susp[I] + bed[I]).sum()
        scale = np.abs(cs[I]).sum() + np.abs(c_old[I] * hh[I]).sum() + np.abs(bed[I]).sum()
        assert np.abs(bed[I]).sum() > 1e-3 * scale      # the bed exchanges sediment
        assert np.abs(susp[I]).sum() > 1e-3 * scale     # and the load moves
        assert abs(ledger) <= tol * scale, (step, ledger, scale)


@pytest.mark.parametrize("precision,tol", [(XBG_FP64, 1e-12), (XBG_FP32, 1e-6)])
def test_sediment_ledger_closes(precision, tol):
    p, zb, bnd = _sed_case()
    m = Model(p, precision)
    _sed_start(m, p, zb, bnd)
    sediment_ledger(m, p, tol)
    m.close()
