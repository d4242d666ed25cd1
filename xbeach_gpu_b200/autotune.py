"""Autotuner of the batched and the single-domain step.

The batched kernels are persistent: each launch runs a chosen number of
blocks that walk contiguous runs of the (scenario, tile) work list of its
tile shape.  The best number depends on the kernel's occupancy, the number of
work items and how ragged the scenarios are, and on which implementation
runs: the wave rows pass has TMA plane tiles with one or two cells per thread
(32 x 8 cells on 256 or 128 threads) and thread-copied tiles; the flow step's
momentum updates run fused into one pass or split in two (a fusion split);
and the passes that read only a cell and its nearest neighbours (wavforce,
the depth/viscosity and momentum passes, the first sediment pass) run in
tiles of 32 x 8 or 64 x 4 cells (two tile shapes, both compiled) or, for one
domain, over row segments of four cells per thread.  They
trade per-item latency, occupancy, per-cell instructions and memory traffic
differently, so all are measured: for each phase, every (kernel variants,
block count) candidate is timed with CUDA events around each kernel of a
batched step (xbg_batch_profile_step), the fastest is kept, and the choice is
cached in a JSON file keyed by (phase, scenario grids, ntheta, precision,
GPU name) so a later batch of the same make-up reuses it.  A single domain
(model.Model) has no persistent blocks: its variants alone are searched, by
the same measurement, and cached by (phase, nx, ny, ntheta, precision, GPU).

    from xbeach_gpu_b200.autotune import tune
    choice = tune(batch)   # applies and returns {shape: blocks, "wave_variant": v, "flow_variant": f, "tile_variant": t}
    choice = tune(model)   # applies and returns {"wave_variant": v, "flow_variant": f, "tile_variant": t}
"""
import hashlib
import json
import os

from .abi import XBG_PHASE_FLOW, XBG_PHASE_TILE, XBG_PHASE_WAVE
from .model import XbgError

# the tile shapes of xbg_batch_set_grid that the phases below launch with
SHAPE_TILE, SHAPE_WROWS, SHAPE_LIN, SHAPE_DT, SHAPE_WIDE = 0, 1, 2, 5, 6
# phases: the tile shape of xbg_batch_set_grid they launch with, the kernels
# timed, and the kernel-variant settings searched, each a tuple of
# (xbg_set_kernel_variant phase, variant) pairs (empty: the phase has one
# form).  The "tile" phase searches the momentum fusion split with the
# pointwise passes' tile shape; with 64 x 4 tiles those passes take the
# 64 x 4 work list, given the same number of persistent blocks; the row
# segments (tile variant 2) are a single-domain form, which a batch refuses.
_T, _F = XBG_PHASE_TILE, XBG_PHASE_FLOW
PHASES = {
    "tile": (SHAPE_TILE, {"k_wave_force", "k_flow_a", "k_flow_u", "k_flow_v", "k_flow_uv", "k_flow_corr",
                          "k_flow_final", "k_sed_a", "k_sed_b", "k_sed_c"},
             (((_F, 1), (_T, 0)), ((_F, 0), (_T, 0)), ((_F, 1), (_T, 1)), ((_F, 0), (_T, 1)),
              ((_F, 1), (_T, 2)), ((_F, 0), (_T, 2)))),
    "wave_rows": (SHAPE_WROWS, {"k_wave_fast", "k_wave_tma"}, (((XBG_PHASE_WAVE, 1),), ((XBG_PHASE_WAVE, 2),),
                                                               ((XBG_PHASE_WAVE, 0),))),
    "lin": (SHAPE_LIN, {"k_disp", "k_means"}, ((),)),
    "dt": (SHAPE_DT, {"k_step_begin"}, ((),)),
}
SHAPES = {sh: (label, kern) for label, (sh, kern, _) in PHASES.items()}
VARIANT_KEY = {XBG_PHASE_WAVE: "wave_variant", XBG_PHASE_FLOW: "flow_variant", XBG_PHASE_TILE: "tile_variant"}
FACTORS = (1, 2, 3, 4, 6, 8, 12, 16)


def _cache_path(path):
    if path:
        return path
    return os.environ.get("XBG_AUTOTUNE_CACHE", os.path.join(os.path.expanduser("~"), ".cache", "xbg_autotune.json"))


def _load(path):
    try:
        with open(path) as f:
            return json.load(f)
    except Exception:
        return {}


def _gpu():
    try:
        import torch
        pr = torch.cuda.get_device_properties(torch.cuda.current_device())
        return pr.name, pr.multi_processor_count
    except Exception:
        return "unknown", 148


def _time_shape(batch, kernels, reps):
    ts = []
    for _ in range(reps):
        prof = batch.profile_step()
        ts.append(sum(t for name, t in prof if name in kernels))
    ts.sort()
    return ts[len(ts) // 2]


def make_up(batch):
    """The batch's make-up in the cache key: scenario grids, ntheta, precision."""
    grids = sorted((m.p.nx, m.p.ny) for m in batch.models)
    h = hashlib.sha1(json.dumps(grids).encode()).hexdigest()[:12]
    prec = "f32" if batch.models[0].dtype.itemsize == 4 else "f64"
    return f"{batch.n}|{h}|{batch.models[0].p.ntheta}|{prec}"


def _apply(target, setting, choice):
    """Set the (phase, variant) pairs of one candidate; False when one does not
    apply to this target."""
    for phase, v in setting:
        try:
            target.set_variant(phase, v)
        except XbgError:
            return False
        choice[VARIANT_KEY[phase]] = v
    return True


def _settings(cached):
    """A cached setting as (phase, variant) pairs (entries are lists of pairs)."""
    return tuple((int(p), int(v)) for p, v in cached)


def tune_model(model, cache=None, reps=3, use_cache=True):
    """Measure and apply the kernel variants of a single domain (a model.Model):
    per phase, every setting is timed over profiled steps and the fastest is
    kept.  Returns {"wave_variant": v, "flow_variant": f, "tile_variant": t}
    (the phases that apply).  The simulation state advances by the profiled
    steps."""
    name, _ = _gpu()
    p = model.p
    prec = "f32" if model.dtype.itemsize == 4 else "f64"
    key0 = f"single|{p.nx}x{p.ny}|{p.ntheta}|{prec}|{name}"
    path = _cache_path(cache)
    db = _load(path) if use_cache else {}
    choice = {}
    for label, (_, kernels, settings) in PHASES.items():
        if settings == ((),):
            continue
        key = f"{label}|{key0}"
        if key in db:
            _apply(model, _settings(db[key]), choice)
            continue
        best = None
        for setting in settings:
            trial = {}
            if not _apply(model, setting, trial):
                continue
            ts = sorted(sum(t for n, t in model.profile_step() if n in kernels) for _ in range(reps))
            t = ts[len(ts) // 2]
            if best is None or t < best[1]:
                best = (setting, t)
        _apply(model, best[0], choice)
        db[key] = [list(x) for x in best[0]]
    if use_cache:
        _save(path, db)
    return choice


def _save(path, db):
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        with open(path, "w") as f:
            json.dump(db, f, indent=1, sort_keys=True)
    except OSError:
        pass


def tune(batch, cache=None, reps=3, shapes=None, use_cache=True):
    """Measure and apply, per phase of `batch` (a model.Batch), the kernel
    variants and the persistent block count.  Returns {shape: blocks} and,
    under "wave_variant", "flow_variant" and "tile_variant", the variants in
    use.  A model.Model is tuned by tune_model.  The simulation state
    advances by the profiled steps."""
    if not hasattr(batch, "set_grid"):
        return tune_model(batch, cache=cache, reps=reps, use_cache=use_cache)
    name, sms = _gpu()
    key0 = f"{make_up(batch)}|{name}"
    path = _cache_path(cache)
    db = _load(path) if use_cache else {}
    choice = {}

    def grid(shape, setting, g):
        batch.set_grid(shape, g)
        if shape == SHAPE_TILE and (XBG_PHASE_TILE, 1) in setting:
            batch.set_grid(SHAPE_WIDE, g)

    for label, (shape, kernels, settings) in PHASES.items():
        if shapes is not None and shape not in shapes:
            continue
        key = f"{label}|{key0}"
        cached = db.get(key)
        if isinstance(cached, list) and len(cached) == 2 and isinstance(cached[0], list):
            setting = _settings(cached[0])
            _apply(batch, setting, choice)
            grid(shape, setting, cached[1])
            choice[shape] = cached[1]
            continue
        best = None
        for setting in settings:
            trial = {}
            if not _apply(batch, setting, trial):   # not available for this batch
                continue
            for f in FACTORS:
                g = sms * f
                grid(shape, setting, g)
                t = _time_shape(batch, kernels, reps)
                if best is None or t < best[2]:
                    best = (setting, g, t)
        setting, g, _ = best
        _apply(batch, setting, choice)
        grid(shape, setting, g)
        choice[shape] = g
        db[key] = [[list(x) for x in setting], g]
    if use_cache:
        _save(path, db)
    return choice
