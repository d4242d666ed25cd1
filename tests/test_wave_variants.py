"""Kernel variants of the same arithmetic.  The wave rows pass has three:
plane tiles moved by the tensor memory accelerator (one box copy per bin,
issued by one thread; the default where it applies) with one or with two
cells per thread, and plane tiles copied by every thread (cp.async).  The
flow step's momentum updates run as one pass (uu* of the tile and its ring
in shared memory) or as two.  The passes that read only a cell and its
nearest neighbours run in 32 x 8 or 64 x 4 blocks.  Each must give the same
state bit for bit over whole coupled steps, on grids whose tiles are partial in x and in y, at the
offshore and lateral edges, for few bins (fewer than the four tile buffers),
with and without the roller, in FP32 and FP64."""
import numpy as np
import pytest

from xbeach_gpu_b200.abi import XBG_FP32, XBG_FP64, XBG_PHASE_FLOW, XBG_PHASE_TILE, XBG_PHASE_WAVE
from xbeach_gpu_b200.model import Model, XbgError
from xbeach_gpu_b200.scenarios import make_case

pytestmark = pytest.mark.gpu

FIELDS = ["ee", "rr", "H", "E", "D", "DR", "R", "thetamean", "Fx", "Fy", "urms", "ust", "zs", "uu", "vv", "zb",
          "C", "hh"]

CASES = {
    "barred_256x128_n18": dict(case="barred_beach", nx=256, ny=128, nt=None, kw={}),
    "linear_200x100_n10": dict(case="linear_beach", nx=200, ny=100, nt=10, kw={}),
    "linear_68x37_n7": dict(case="linear_beach", nx=68, ny=37, nt=7, kw={}),
    "linear_96x12_n3": dict(case="linear_beach", nx=96, ny=12, nt=3, kw={}),
    "linear_64x9_n1": dict(case="linear_beach", nx=64, ny=9, nt=1, kw={}),
    "barred_160x72_noroller": dict(case="barred_beach", nx=160, ny=72, nt=None, kw=dict(roller=0)),
    "linear_100x50_baldock": dict(case="linear_beach", nx=100, ny=50, nt=10, kw=dict(breakmodel=2)),
}


def _model(c, precision, variant, phase=XBG_PHASE_WAVE):
    p, zb, bnd = make_case(c["case"], nx=c["nx"], ny=c["ny"], ntheta=c["nt"])
    for k, v in c["kw"].items():
        setattr(p, k, v)
    m = Model(p, precision)
    m.set_wave_boundary(0, bnd["St"], bnd["q"], t0=0.0, tend=p.rtlength, Trep=bnd["Trep"])
    m.set_sealevel([0.0, 1e6], [0.0, 0.0], [0.0, 0.0])
    m.set_wind([0.0, 1e6], [0.0, 0.0], [0.0, 0.0])
    m.init_state(zb, 0.0, 0.0)
    m.set_variant(phase, variant)
    return m


@pytest.mark.parametrize("precision", [XBG_FP32, XBG_FP64])
@pytest.mark.parametrize("name", sorted(CASES))
def test_tma_tiles_equal_thread_copied_tiles(name, precision):
    c = CASES[name]
    runs = []
    for variant in (0, 1, 2):
        m = _model(c, precision, variant)
        assert m.variant(XBG_PHASE_WAVE) == variant
        m.advance(25)
        m.advance(15)
        t, dt, n, _, rc = m.time()
        assert rc == 0 and n == 40
        runs.append((t, dt, {f: m.get(f).copy() for f in FIELDS}))
        m.close()
    for r in runs[1:]:
        assert runs[0][:2] == r[:2]
        for f in FIELDS:
            assert np.array_equal(runs[0][2][f], r[2][f]), f


# grids whose ny - 2 is a multiple of the tile height put row ny - 3 (the
# vvlatbnd source of row ny - 2) outside the fused pass's shared rows
FLOW_CASES = dict(CASES, linear_70x42_n4=dict(case="linear_beach", nx=70, ny=42, nt=4, kw={}),
                  barred_96x34_n18=dict(case="barred_beach", nx=96, ny=34, nt=None, kw={}))


@pytest.mark.parametrize("precision", [XBG_FP32, XBG_FP64])
@pytest.mark.parametrize("name", sorted(FLOW_CASES))
def test_fused_momentum_pass_equals_two_passes(name, precision):
    c = FLOW_CASES[name]
    runs = []
    for variant in (0, 1):
        m = _model(c, precision, variant, XBG_PHASE_FLOW)
        assert m.variant(XBG_PHASE_FLOW) == variant
        m.advance(25)
        m.advance(15)
        t, dt, n, _, rc = m.time()
        assert rc == 0 and n == 40
        runs.append((t, dt, {f: m.get(f).copy() for f in FIELDS}))
        m.close()
    assert runs[0][:2] == runs[1][:2]
    for f in FIELDS:
        assert np.array_equal(runs[0][2][f], runs[1][2][f]), f


# grids that leave partial 64 x 4 tiles in x and in y, and a sediment case
TILE_CASES = dict(FLOW_CASES, linear_130x45_n5=dict(case="linear_beach", nx=130, ny=45, nt=5, kw={}),
                  sediment_96x38=dict(case="linear_beach", nx=96, ny=38, nt=6,
                                      kw=dict(sedtrans=1, morfac=10.0, sedstart=0.0)))


@pytest.mark.parametrize("precision", [XBG_FP32, XBG_FP64])
@pytest.mark.parametrize("name", sorted(TILE_CASES))
def test_wide_tiles_equal_narrow_tiles(name, precision):
    """Variants 0 and 1: 32 x 8 and 64 x 4 blocks; 2: row segments with
    16-byte loads (where nx is a multiple of the segment width; refused
    elsewhere)."""
    c = TILE_CASES[name]
    runs = []
    seg = 4 if precision == XBG_FP32 else 2
    for variant in (0, 1, 2):
        if variant == 2 and c["nx"] % seg:
            with pytest.raises(XbgError):
                _model(c, precision, variant, XBG_PHASE_TILE)
            continue
        m = _model(c, precision, variant, XBG_PHASE_TILE)
        assert m.variant(XBG_PHASE_TILE) == variant
        m.advance(25)
        m.advance(15)
        t, dt, n, _, rc = m.time()
        assert rc == 0 and n == 40
        runs.append((t, dt, {f: m.get(f).copy() for f in FIELDS}))
        m.close()
    for r in runs[1:]:
        assert runs[0][:2] == r[:2]
        for f in FIELDS:
            assert np.array_equal(runs[0][2][f], r[2][f]), f


def test_single_domain_autotune(tmp_path):
    """The single-domain autotuner measures each phase's variants, applies the
    fastest and caches it; a second call reuses the cache.  The results do
    not depend on the choice."""
    from xbeach_gpu_b200.autotune import tune
    c = CASES["barred_256x128_n18"]
    ref = _model(c, XBG_FP32, 1)
    ref.advance(12)
    want = {f: ref.get(f).copy() for f in FIELDS}
    ref.close()
    m = _model(c, XBG_FP32, 1)
    cache = str(tmp_path / "tune.json")
    choice = tune(m, cache=cache, reps=1)
    assert set(choice) == {"wave_variant", "flow_variant", "tile_variant"}
    assert m.variant(XBG_PHASE_WAVE) == choice["wave_variant"]
    assert m.variant(XBG_PHASE_FLOW) == choice["flow_variant"]
    assert m.variant(XBG_PHASE_TILE) == choice["tile_variant"]
    _, _, n, _, rc = m.time()
    assert rc == 0 and 0 < n < 12
    m.advance(12 - n)
    for f in FIELDS:
        assert np.array_equal(m.get(f), want[f]), f
    m2 = _model(c, XBG_FP32, 1)
    assert tune(m2, cache=cache, reps=1) == choice
    _, _, n2, _, _ = m2.time()
    assert n2 == 0   # from the cache: nothing profiled
    m.close()
    m2.close()


def test_tma_variant_applies_only_where_it_can():
    """nx not a multiple of 4 (row pitch of a tensor map) or wave-current
    interaction on: the thread-copied tiles, and asking for the TMA ones is
    refused."""
    for nx, kw in ((45, {}), (64, dict(wci=1.0, hwci=0.5))):
        p, zb, bnd = make_case("linear_beach", nx=nx, ny=32, ntheta=6)
        for k, v in kw.items():
            setattr(p, k, v)
        m = Model(p)
        assert m.variant(XBG_PHASE_WAVE) == 0
        for v in (1, 2):
            with pytest.raises(XbgError):
                m.set_variant(XBG_PHASE_WAVE, v)
        m.close()
    p, zb, bnd = make_case("linear_beach", nx=64, ny=32, ntheta=6)
    m = Model(p)
    assert m.variant(XBG_PHASE_WAVE) == 1
    m.close()


def test_negative_energy_is_clipped_when_set():
    """The wave pass relies on ee >= 0 in memory (its sanity step); a caller
    that sets negative values gets them clipped, as that step would."""
    p, zb, bnd = make_case("linear_beach", nx=64, ny=32, ntheta=6)
    m = Model(p)
    ee = np.linspace(-5.0, 5.0, p.nx * p.ny * p.ntheta).astype(np.float32)
    m.set("ee", ee)
    assert np.array_equal(m.get("ee"), np.maximum(ee, 0.0))
    m.close()
