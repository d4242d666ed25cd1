"""Autotuner of the batched step.

The batched kernels are persistent: each launch runs a chosen number of
blocks that walk contiguous runs of the (scenario, tile) work list of its
tile shape.  The best number depends on the kernel's occupancy, the number of
work items and how ragged the scenarios are, and on which implementation
runs: the wave rows pass has TMA plane tiles with one or two cells per thread
(tile shapes of 32 x 8 cells on 256 or 128 threads) and thread-copied tiles,
and the flow step's momentum updates run fused into one pass or split in two
(a fusion split).  They trade per-item latency, occupancy, per-cell
instructions and memory traffic differently, so all are measured: for each
phase, every (kernel variant, block count) candidate is timed with CUDA
events around each kernel of a batched step (xbg_batch_profile_step), the
fastest is kept, and the choice is cached in a JSON file keyed by (phase,
scenario grids, ntheta, precision, GPU name) so a later batch of the same
make-up reuses it.

    from xbeach_gpu_b200.autotune import tune
    choice = tune(batch)   # applies and returns {shape: blocks, "wave_variant": v, "flow_variant": f}
"""
import hashlib
import json
import os

from .abi import XBG_PHASE_FLOW, XBG_PHASE_WAVE
from .model import XbgError

# phases: the tile shape of xbg_batch_set_grid they launch with, the kernels
# timed, the xbg_set_kernel_variant phase and the variants searched (None:
# the phase has one)
PHASES = {
    "tile": (0, {"k_wave_force", "k_flow_a", "k_flow_u", "k_flow_v", "k_flow_uv", "k_flow_corr", "k_flow_final",
                 "k_sed_a", "k_sed_b", "k_sed_c"}, XBG_PHASE_FLOW, (1, 0)),
    "wave_rows": (1, {"k_wave_fast", "k_wave_tma"}, XBG_PHASE_WAVE, (1, 2, 0)),
    "lin": (2, {"k_disp", "k_means"}, None, (None,)),
    "dt": (5, {"k_step_begin"}, None, (None,)),
}
SHAPES = {sh: (label, kern) for label, (sh, kern, _, _) in PHASES.items()}
VARIANT_KEY = {XBG_PHASE_WAVE: "wave_variant", XBG_PHASE_FLOW: "flow_variant"}
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


def tune(batch, cache=None, reps=3, shapes=None, use_cache=True):
    """Measure and apply, per phase of `batch` (a model.Batch), the kernel
    variant and the persistent block count.  Returns {shape: blocks} and,
    under "wave_variant" and "flow_variant", the variants in use.  The
    simulation state advances by the profiled steps."""
    name, sms = _gpu()
    key0 = f"{make_up(batch)}|{name}"
    path = _cache_path(cache)
    db = _load(path) if use_cache else {}
    choice = {}
    for label, (shape, kernels, vphase, variants) in PHASES.items():
        if shapes is not None and shape not in shapes:
            continue
        key = f"{label}|{key0}"
        if key in db:
            v, g = db[key]
            if v is not None:
                batch.set_variant(vphase, v)
                choice[VARIANT_KEY[vphase]] = v
            batch.set_grid(shape, g)
            choice[shape] = g
            continue
        best = None
        for v in variants:
            if v is not None:
                try:
                    batch.set_variant(vphase, v)
                except XbgError:   # not available for this batch
                    continue
            for f in FACTORS:
                g = sms * f
                batch.set_grid(shape, g)
                t = _time_shape(batch, kernels, reps)
                if best is None or t < best[2]:
                    best = (v, g, t)
        v, g, _ = best
        if v is not None:
            batch.set_variant(vphase, v)
            choice[VARIANT_KEY[vphase]] = v
        batch.set_grid(shape, g)
        choice[shape] = g
        db[key] = [v, g]
    if use_cache:
        try:
            os.makedirs(os.path.dirname(path), exist_ok=True)
            with open(path, "w") as f:
                json.dump(db, f, indent=1, sort_keys=True)
        except OSError:
            pass
    return choice
