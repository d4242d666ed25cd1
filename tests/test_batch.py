"""Batched scenarios (xbg_batch_*) against the same scenarios stepped one by
one through the single-domain handle.

The batched kernels run the single-domain kernels' bodies on each scenario's
tiles, the dt reduction is a min (order-free) and the ubnd column sum keeps
the single-domain thread count, so every scenario must come out bit for bit
the same, with its own dt and step count."""
import numpy as np
import pytest

from xbeach_gpu_b200.abi import XBG_FLAG_ENDED, XBG_FP32, XBG_FP64
from xbeach_gpu_b200.model import Batch, Model
from xbeach_gpu_b200.scenarios import make_ensemble

pytestmark = pytest.mark.gpu

FIELDS = ["zs", "uu", "vv", "hh", "zb", "H", "E", "D", "DR", "Fx", "Fy", "urms", "ust", "C", "ee", "rr",
          "ueu", "vev", "hu", "hv", "qx", "qy", "stdep", "Hmean", "zsmax"]


def _setup(m, p, zb, bnd):
    m.set_wave_boundary(0, bnd["St"], bnd["q"], t0=0.0, tend=p.rtlength, Trep=bnd["Trep"])
    m.set_sealevel([0.0, 1e6], [0.0, 0.0], [0.0, 0.0])
    m.set_wind([0.0, 1e6], [0.0, 0.0], [0.0, 0.0])
    m.init_state(zb, 0.0, 0.0)


def _cases(n, seed):
    return make_ensemble(n, seed=seed, nx_range=(64, 192), ny_range=(32, 96), dtbc=5.0)


@pytest.mark.parametrize("precision", [XBG_FP32, XBG_FP64])
def test_batch_matches_single_domain(precision):
    sc = _cases(5, 11)
    b = Batch([p for p, _, _ in sc], precision)
    for s, (p, zb, bnd) in enumerate(sc):
        _setup(b.scenario(s), p, zb, bnd)
    b.advance(30)
    b.advance(30)
    st = b.status()
    assert len(set(int(v) for v in st["nstep"])) == 1 and st["nstep"][0] == 60
    assert len(set(float(v) for v in st["dt"])) > 1   # each scenario its own dt
    for s, (p, zb, bnd) in enumerate(sc):
        m = Model(p, precision)
        _setup(m, p, zb, bnd)
        m.advance(60)
        t, dt, n, fl, rc = m.time()
        assert rc == 0 and st["status"][s] == 0
        assert (st["nstep"][s], st["t"][s], st["dt"][s]) == (n, t, dt), s
        for f in FIELDS:
            assert np.array_equal(b.scenario(s).get(f), m.get(f)), (s, f)
        m.close()
    b.close()


def test_batch_scenarios_end_on_their_own():
    """A scenario that reaches its end time stops; the others go on, and are
    still identical to their single-domain runs."""
    sc = _cases(3, 5)
    sc[1][0].endtime = 5.0
    b = Batch([p for p, _, _ in sc], XBG_FP32)
    for s, (p, zb, bnd) in enumerate(sc):
        _setup(b.scenario(s), p, zb, bnd)
    b.advance(80)
    st = b.status()
    assert st["flags"][1] & XBG_FLAG_ENDED and abs(st["t"][1] - 5.0) < 1e-9
    assert not (st["flags"][0] & XBG_FLAG_ENDED) and st["t"][0] > 5.0
    p, zb, bnd = sc[2]
    m = Model(p, XBG_FP32)
    _setup(m, p, zb, bnd)
    m.advance(80)
    assert m.time()[2] == st["nstep"][2]
    for f in ["zs", "uu", "H", "zb", "ee"]:
        assert np.array_equal(b.scenario(2).get(f), m.get(f)), f
    m.close()
    b.close()


def test_batch_grid_choice_does_not_change_results(tmp_path):
    """The autotuner's knobs (persistent blocks per tile shape, the wave rows
    variant, the flow pass split) only change which block runs which tile,
    how the tiles are moved and where the passes cut: batches with different
    block counts and any of the variants end bit for bit the same."""
    from xbeach_gpu_b200.autotune import tune
    sc = _cases(4, 21)
    from xbeach_gpu_b200.abi import XBG_PHASE_FLOW, XBG_PHASE_TILE, XBG_PHASE_WAVE
    runs = []
    for variant in ("default", "tuned", "thread_tiles", "two_cells", "other_flow_split", "wide_tiles"):
        b = Batch([p for p, _, _ in sc], XBG_FP32)
        for s, (p, zb, bnd) in enumerate(sc):
            _setup(b.scenario(s), p, zb, bnd)
        if variant == "tuned":
            for shape, blocks in ((0, 7), (1, 3), (2, 5), (5, 2)):
                b.set_grid(shape, blocks)
        if variant == "thread_tiles":
            assert b.variant(XBG_PHASE_WAVE) == 1
            b.set_variant(XBG_PHASE_WAVE, 0)
            assert b.variant(XBG_PHASE_WAVE) == 0
        if variant == "two_cells":
            b.set_variant(XBG_PHASE_WAVE, 2)
            assert b.variant(XBG_PHASE_WAVE) == 2
        if variant == "other_flow_split":
            f = 1 - b.variant(XBG_PHASE_FLOW)
            b.set_variant(XBG_PHASE_FLOW, f)
            assert b.variant(XBG_PHASE_FLOW) == f
        if variant == "wide_tiles":
            b.set_variant(XBG_PHASE_TILE, 1)
            assert b.variant(XBG_PHASE_TILE) == 1
            b.set_grid(6, 5)
        b.advance(25)
        runs.append({s: {f: b.scenario(s).get(f).copy() for f in ("zs", "uu", "H", "ee")} for s in range(len(sc))})
        if variant == "tuned":
            choice = tune(b, cache=str(tmp_path / "tune.json"), reps=1)
            assert {0, 1, 2, 5} <= set(choice) and all(choice[k] >= 1 for k in (0, 1, 2, 5))
            assert choice["tile_variant"] in (0, 1) and b.variant(XBG_PHASE_TILE) == choice["tile_variant"]
            assert choice["wave_variant"] in (0, 1, 2) and b.variant(XBG_PHASE_WAVE) == choice["wave_variant"]
            assert choice["flow_variant"] in (0, 1) and b.variant(XBG_PHASE_FLOW) == choice["flow_variant"]
            again = tune(b, cache=str(tmp_path / "tune.json"), reps=1)   # from the cache
            assert again == choice
        b.close()
    for s in runs[0]:
        for f in runs[0][s]:
            for r in runs[1:]:
                assert np.array_equal(runs[0][s][f], r[s][f]), (s, f)
