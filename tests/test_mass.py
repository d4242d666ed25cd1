"""Water mass balance of the CUDA flow step.

Continuity (Flow_kernel.cu:1626-1681) and the second-order water-level
correction (wrkzs2Ocorr / zs2Ocorr, :2130-2317, which also adds its fluxes to
qx and qy) are together a flux-form update: for every cell with ix >= 1 and
1 <= iy <= ny-2,
    zs_new - zs_old = dt/dx (QX[ix-1] - QX[ix] + QY[iy-1] - QY[iy])
with the step's final fluxes QX, QY.  Summed over those cells the volume
change is the flux through the domain's faces; the lateral rows (latbnd) and
the offshore column (ubnd1D) are copies, i.e. sources by the reference's
design, and are reported separately.  The ledger closes to 1e-12 of the water
volume in FP64 and to 1e-6 in FP32."""
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
