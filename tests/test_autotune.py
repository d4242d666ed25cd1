"""The autotuner's search and cache logic, on fake targets (no GPU): every
(kernel variants, block count) candidate of a phase is timed, the fastest is
applied and cached, a cached choice is applied without timing, a variant the
target refuses is skipped, a cache entry of another format is measured
again, and a single domain is tuned over its variants alone."""
import json

import pytest

from xbeach_gpu_b200 import autotune as at
from xbeach_gpu_b200.abi import XBG_PHASE_FLOW, XBG_PHASE_TILE, XBG_PHASE_WAVE
from xbeach_gpu_b200.model import XbgError


class _P:
    def __init__(self, nx, ny, ntheta=12):
        self.nx, self.ny, self.ntheta = nx, ny, ntheta


class _DType:
    itemsize = 4


class FakeModel:
    """Times each kernel of a profiled step from the variants in use; refuses
    the variants listed in `refuse`."""

    dtype = _DType()

    def __init__(self, nx=256, ny=128, best=None, refuse=()):
        self.p = _P(nx, ny)
        self.var = {XBG_PHASE_WAVE: 1, XBG_PHASE_FLOW: 0, XBG_PHASE_TILE: 0}
        self.best = best or {XBG_PHASE_WAVE: 2, XBG_PHASE_FLOW: 1, XBG_PHASE_TILE: 1}
        self.refuse = set(refuse)
        self.steps = 0

    def set_variant(self, phase, v):
        if (phase, v) in self.refuse:
            raise XbgError("refused")
        self.var[phase] = v

    def variant(self, phase):
        return self.var[phase]

    def _cost(self, phases):
        return sum(0.0 if self.var[p] == self.best[p] else 1.0 for p in phases)

    def profile_step(self):
        self.steps += 1
        tile = 1.0 + self._cost((XBG_PHASE_FLOW, XBG_PHASE_TILE))
        return [("k_flow_corr", tile), ("k_wave_tma", 1.0 + self._cost((XBG_PHASE_WAVE,))), ("k_disp", 0.5)]


class FakeBatch(FakeModel):
    """A batch adds persistent block counts per tile shape; the tile kernels
    are fastest at `best_blocks` on the shape they run on."""

    def __init__(self, best_blocks=148 * 4, **kw):
        kw.setdefault("refuse", {(XBG_PHASE_TILE, 2)})   # row segments are a single-domain form
        super().__init__(**kw)
        self.models = [FakeModel(nx, ny) for nx, ny in ((256, 128), (512, 256))]
        self.n = len(self.models)
        self.grid = {}
        self.best_blocks = best_blocks

    def set_grid(self, shape, blocks):
        self.grid[shape] = blocks

    def profile_step(self):
        self.steps += 1
        shape = at.SHAPE_WIDE if self.var[XBG_PHASE_TILE] == 1 else at.SHAPE_TILE
        blocks = abs(self.grid.get(shape, 0) - self.best_blocks) / self.best_blocks
        tile = 1.0 + self._cost((XBG_PHASE_FLOW, XBG_PHASE_TILE)) + blocks
        wave = 1.0 + self._cost((XBG_PHASE_WAVE,)) + abs(self.grid.get(at.SHAPE_WROWS, 0) - 296) / 296
        return [("k_flow_corr", tile), ("k_wave_tma", wave), ("k_disp", 0.5), ("k_step_begin", 0.1)]


@pytest.fixture(autouse=True)
def _gpu(monkeypatch):
    monkeypatch.setattr(at, "_gpu", lambda: ("fake", 148))


def test_batch_search_applies_and_caches(tmp_path):
    cache = str(tmp_path / "tune.json")
    b = FakeBatch()
    choice = at.tune(b, cache=cache, reps=1)
    assert choice["wave_variant"] == 2 and choice["flow_variant"] == 1 and choice["tile_variant"] == 1
    assert b.var == {XBG_PHASE_WAVE: 2, XBG_PHASE_FLOW: 1, XBG_PHASE_TILE: 1}
    assert choice[at.SHAPE_TILE] == 148 * 4 and b.grid[at.SHAPE_WIDE] == 148 * 4
    assert choice[at.SHAPE_WROWS] == 296
    db = json.load(open(cache))
    assert any(k.startswith("tile|") for k in db) and any(k.startswith("wave_rows|") for k in db)
    # the cached choice is applied to a batch of the same make-up without timing
    b2 = FakeBatch()
    assert at.tune(b2, cache=cache, reps=1) == choice
    assert b2.steps == 0 and b2.var == b.var and b2.grid[at.SHAPE_WIDE] == 148 * 4


def test_refused_variant_is_skipped(tmp_path):
    b = FakeBatch(refuse={(XBG_PHASE_WAVE, 2), (XBG_PHASE_TILE, 2)},
                  best={XBG_PHASE_WAVE: 2, XBG_PHASE_FLOW: 0, XBG_PHASE_TILE: 0})
    choice = at.tune(b, cache=str(tmp_path / "t.json"), reps=1)
    assert choice["wave_variant"] in (0, 1) and choice["flow_variant"] == 0 and choice["tile_variant"] == 0
    assert b.var[XBG_PHASE_TILE] == 0 and b.grid[at.SHAPE_TILE] == 148 * 4


def test_cache_entry_of_another_format_is_measured_again(tmp_path):
    cache = tmp_path / "tune.json"
    b = FakeBatch()
    key = f"tile|{at.make_up(b)}|fake"
    cache.write_text(json.dumps({key: [1, 444]}))
    choice = at.tune(b, cache=str(cache), reps=1)
    assert b.steps > 0 and choice[at.SHAPE_TILE] == 148 * 4
    assert json.loads(cache.read_text())[key] == [[[XBG_PHASE_FLOW, 1], [XBG_PHASE_TILE, 1]], 148 * 4]


def test_single_domain_search(tmp_path):
    cache = str(tmp_path / "tune.json")
    m = FakeModel()
    choice = at.tune(m, cache=cache, reps=1)
    assert choice == {"wave_variant": 2, "flow_variant": 1, "tile_variant": 1}
    assert m.steps == 6 + 3   # six tile-phase settings and three wave variants, one step each
    m2 = FakeModel()
    assert at.tune(m2, cache=cache, reps=1) == choice and m2.steps == 0
    m4 = FakeModel(best={XBG_PHASE_WAVE: 1, XBG_PHASE_FLOW: 0, XBG_PHASE_TILE: 2})
    assert at.tune(m4, cache=str(tmp_path / "t4.json"), reps=1)["tile_variant"] == 2
    # another grid is another cache key
    m3 = FakeModel(nx=512)
    at.tune(m3, cache=cache, reps=1)
    assert m3.steps == 9
