"""xbg_flow_dt_noalloc, the entry point that allocates no device memory.

Some callers cannot allocate on the device: a coupler or framework that has
handed the GPU's memory to its own pool allocator, or a caller whose other
streams must not be stalled by the device-wide synchronisation of
cudaMalloc/cudaFree.  They own the water depth and the output; the entry
point's only scratch is a fixed array inside the library.  These tests call
it through the C ABI on caller-owned device buffers and compare its result
with the dt that the existing entry point xbg_compute_dt derives from the
same depths, on two calls in a row (a large grid, then a small one whose
minimum is larger, so stale block minima left by the first call would show).

The dt limiter and output-time snapping of xbg_compute_dt are kept out of the
way (previous dt equal to the expected one, output and end times far off), so
both give 0.5 * min(cfl*dx/sqrt(9.81*hh)) from the same maximum depth and the
same single square root; what remains is xbg_compute_dt's snapping of dt to
a whole number of steps before the output time (1e12 s away), a relative
change below 1e-12, hence the 1e-9 tolerance in both precisions.
"""
import numpy as np
import pytest

from helpers import small_params
from xbeach_gpu_b200.abi import XBG_FP32, XBG_FP64
from xbeach_gpu_b200.model import Model, load

pytestmark = pytest.mark.gpu

TOL = {XBG_FP32: 1e-9, XBG_FP64: 1e-9}
XBG_ERR_ARG = 1


def _case(nx, ny, hmax, precision, seed):
    p, _ = small_params(nx, ny, 6, swave=0, outputtimestep=1e12, endtime=2e12)
    dt = np.float32 if precision == XBG_FP32 else np.float64
    hh = np.random.default_rng(seed).uniform(0.02, hmax, nx * ny).astype(dt)
    return p, hh


def _compute_dt(p, hh, precision):
    m = Model(p, precision)
    m.set("hh", hh)
    guess = 0.5 * float(np.min(p.CFL * p.dx / np.sqrt(9.81 * hh.astype(np.float64))))
    m.set_time(0.0, guess, guess)
    m.compute_dt()
    t, dt, _, _, rc = m.time()
    assert rc == 0
    m.close()
    return dt


@pytest.mark.parametrize("precision", [XBG_FP32, XBG_FP64])
def test_noalloc_matches_compute_dt_twice(precision):
    import torch
    L = load()
    tdt = torch.float32 if precision == XBG_FP32 else torch.float64
    cases = [_case(700, 500, 12.0, precision, 11), _case(77, 53, 2.0, precision, 12)]
    stream = torch.cuda.Stream()
    bufs = [(torch.from_numpy(hh).cuda(), torch.full((1,), -1.0, dtype=tdt, device="cuda")) for _, hh in cases]
    warm = torch.full((1,), -1.0, dtype=tdt, device="cuda")
    torch.cuda.synchronize()
    # a first call (the array's address lookup, the module load), then the
    # device's free memory must not change over the calls under test
    (p0, _), (h0, _) = cases[1], bufs[1]
    assert L.xbg_flow_dt_noalloc(precision, h0.data_ptr(), p0.nx, p0.ny, p0.dx, p0.CFL, warm.data_ptr(),
                                 stream.cuda_stream) == 0
    stream.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for (p, _), (hd, out) in zip(cases, bufs):      # two calls in a row, same stream
        rc = L.xbg_flow_dt_noalloc(precision, hd.data_ptr(), p.nx, p.ny, p.dx, p.CFL, out.data_ptr(),
                                   stream.cuda_stream)
        assert rc == 0
    stream.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    got = [float(out.cpu()[0]) for _, out in bufs]
    assert got[0] < got[1]
    for (p, hh), g in zip(cases, got):
        want = _compute_dt(p, hh, precision)
        assert abs(g - want) <= TOL[precision] * want, (g, want)


def test_noalloc_rejects_oversize_grid():
    """Grids above XBG_NOALLOC_MAX_CELLS are refused before any device work:
    the argument check comes first, so the small buffer passed with the
    oversize grid is never read."""
    import torch
    L = load()
    n = (1 << 30) + 1
    hd = torch.ones(16, dtype=torch.float32, device="cuda")
    out = torch.full((1,), -1.0, dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    assert L.xbg_flow_dt_noalloc(XBG_FP32, hd.data_ptr(), n, 1, 4.0, 0.7, out.data_ptr(), None) == XBG_ERR_ARG
    assert L.xbg_flow_dt_noalloc(XBG_FP32, hd.data_ptr(), 0, 1, 4.0, 0.7, out.data_ptr(), None) == XBG_ERR_ARG
    assert L.xbg_flow_dt_noalloc(XBG_FP32, hd.data_ptr(), 1, 1, 4.0, 0.7, None, None) == XBG_ERR_ARG
    torch.cuda.synchronize()
    assert float(out.cpu()[0]) == -1.0


@pytest.mark.parametrize("precision", [XBG_FP32, XBG_FP64])
def test_noalloc_reports_nonfinite_depth(precision):
    """A NaN depth makes the result NaN (a caller testing dt > 0 sees it)
    instead of being skipped by the minimum; the next call on clean depths
    is unaffected."""
    import torch
    L = load()
    tdt = torch.float32 if precision == XBG_FP32 else torch.float64
    hh = torch.full((300 * 200,), 3.0, dtype=tdt, device="cuda")
    hh[12345] = float("nan")
    out = torch.zeros(2, dtype=tdt, device="cuda")
    assert L.xbg_flow_dt_noalloc(precision, hh.data_ptr(), 300, 200, 4.0, 0.7, out.data_ptr(), None) == 0
    hh[12345] = 3.0
    assert L.xbg_flow_dt_noalloc(precision, hh.data_ptr(), 300, 200, 4.0, 0.7, out.data_ptr() + out.element_size(),
                                 None) == 0
    torch.cuda.synchronize()
    r = out.cpu().numpy()
    assert np.isnan(r[0])
    assert abs(r[1] - 0.5 * 0.7 * 4.0 / np.sqrt(9.81 * 3.0)) <= 1e-6 * r[1]
