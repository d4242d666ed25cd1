"""Autotuner of the batched step.

The batched kernels are persistent: each launch runs a chosen number of
blocks that walk contiguous runs of the (scenario, tile) work list of its
tile shape.  The best number depends on the kernel's occupancy, the number of
work items and how ragged the scenarios are, so it is measured: for each
shape, every candidate block count is timed with CUDA events around each
kernel of a batched step (xbg_batch_profile_step), the fastest is kept, and
the choice is cached in a JSON file keyed by (shape, scenarios, cells,
ntheta, precision, GPU name) so a later batch of the same make-up reuses it.

    from xbeach_gpu_b200.autotune import tune
    choice = tune(batch)          # applies and returns {shape: blocks}
"""
import json
import os

# tile shapes of xbg_batch_set_grid and the kernels that use them
SHAPES = {
    0: ("tile", {"k_wave_force", "k_flow_a", "k_flow_u", "k_flow_v", "k_flow_corr",
                 "k_flow_final", "k_sed_a", "k_sed_b", "k_sed_c"}),
    1: ("wave_rows", {"k_wave_fast"}),
    2: ("lin", {"k_disp", "k_means"}),
    5: ("dt", {"k_step_begin"}),
}
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


def tune(batch, cache=None, reps=3, shapes=None, use_cache=True):
    """Measure and apply the persistent block count of each tile shape of
    `batch` (a model.Batch).  Returns {shape: blocks}.  The simulation state
    advances by the profiled steps."""
    name, sms = _gpu()
    cells = sum(m.p.nx * m.p.ny for m in batch.models)
    nt = batch.models[0].p.ntheta
    prec = "f32" if batch.models[0].dtype.itemsize == 4 else "f64"
    path = _cache_path(cache)
    db = _load(path) if use_cache else {}
    choice = {}
    for shape in (shapes or SHAPES):
        label, kernels = SHAPES[shape]
        key = f"{label}|{batch.n}|{cells}|{nt}|{prec}|{name}"
        if key in db:
            choice[shape] = int(db[key])
            batch.set_grid(shape, choice[shape])
            continue
        best = None
        for f in FACTORS:
            g = sms * f
            batch.set_grid(shape, g)
            t = _time_shape(batch, kernels, reps)
            if best is None or t < best[1]:
                best = (g, t)
        choice[shape] = best[0]
        batch.set_grid(shape, best[0])
        db[key] = best[0]
    if use_cache:
        try:
            os.makedirs(os.path.dirname(path), exist_ok=True)
            with open(path, "w") as f:
                json.dump(db, f, indent=1, sort_keys=True)
        except OSError:
            pass
    return choice
