"""Coupled cell-updates/s of the XBeach_GPU coupled step on B200.

Workload: the large single domain (barred beach, nx=2048 x ny=1024, dx=2 m,
18 directional bins over -90..90 deg, JONSWAP-shaped wave-group forcing,
sediment with morfac 10), FP32, seeded synthetic inputs.  One step = one
whole coupled timestep (dt, boundaries, wave action, shallow-water flow,
sediment and bed, running means) over every cell, replayed from the CUDA
graph of libxbg_b200.so.  Multi-GPU: independent replicas (the path has no
exchange step), value = cells * steps * ranks / max-over-ranks time.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Prints one JSON line (rank 0).
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

B_ALGO = lambda nt: 4 * (77 + 4 * nt)   # algorithmic bytes per coupled cell-update

# DRAM bytes (read + write) per launch of the dominant kernel, from one ncu
# capture of this workload (dram__bytes_read.sum + dram__bytes_write.sum; the
# capture and its command are summarised under profiles/).  Keyed by
# (kernel, nx, ny, ntheta); other workloads report traffic null.
NCU_TRAFFIC = {
    ("k_wave_fast", 2048, 1024, 18): 361049088 + 335545344,
    ("k_wave_tma", 2048, 1024, 18): 345307392 + 328110592,
}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--nx", type=int, default=2048)
    ap.add_argument("--ny", type=int, default=1024)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="large", choices=["large", "ensemble", "surrogate", "storm"],
                    help="large: the 2048x1024 single domain (the headline line); ensemble: the batched "
                         "ragged ensemble (256 scenarios, one launch per kernel for all); storm: the "
                         "surrogate-assisted storm ensemble (512 scenarios) beside its plain run")
    ap.add_argument("--no-extras", action="store_true",
                    help="large: leave out the ensemble and storm-ensemble keys of the line")
    ap.add_argument("--storm-scenarios", type=int, default=512)
    ap.add_argument("--storm-steps", type=int, default=100)
    ap.add_argument("--scenarios", type=int, default=256)
    ap.add_argument("--no-autotune", action="store_true", help="ensemble: keep the default persistent grids")
    ap.add_argument("--surrogate-base", type=int, default=32, choices=[16, 32],
                    help="surrogate: channels of the U-Net's first level")
    return ap.parse_args()


def over_ranks(dist, maxed, summed, device):
    """Max over ranks of `maxed` (times) and sum of `summed` (work), one
    all-reduce each; every rank calls it with lists of the same lengths."""
    import torch
    mx = torch.tensor([float(v) for v in maxed], device=device, dtype=torch.float64)
    sm = torch.tensor([float(v) for v in summed], device=device, dtype=torch.float64)
    if dist is not None:
        dist.all_reduce(mx, op=dist.ReduceOp.MAX)
        dist.all_reduce(sm, op=dist.ReduceOp.SUM)
    return [float(v) for v in mx], [float(v) for v in sm]


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class NvmlClockSampler:
    """SM clock, its maximum, power and the clock-event (throttle) reasons
    read through NVML (the library nvidia-smi reports from) every 2 ms on a
    background thread, so that even a timed region of a few tens of
    milliseconds holds several samples; stop() keeps those inside
    [mark_start(), mark_end()]."""
    REASONS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40), ("sw_thermal_slowdown", 0x20),
               ("sw_power_cap", 0x4))

    def __init__(self, local):
        import pynvml
        self.nv = pynvml
        pynvml.nvmlInit()
        h = None
        try:
            import torch
            uuid = str(torch.cuda.get_device_properties(local).uuid)
            h = pynvml.nvmlDeviceGetHandleByUUID(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
        except Exception:
            h = pynvml.nvmlDeviceGetHandleByIndex(local)
        self.h = h
        self.rows = []
        self.t0 = self.t1 = None
        self.run = False

    def start(self):
        self.run = True
        self.th = threading.Thread(target=self._loop, daemon=True)
        self.th.start()

    def _loop(self):
        nv, h = self.nv, self.h
        mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
        while self.run:
            try:
                sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                rs = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                pw = nv.nvmlDeviceGetPowerUsage(h) / 1000.0
                self.rows.append((time.time(), sm, mx, rs, pw))
            except Exception:
                pass
            time.sleep(0.002)

    def mark_start(self):
        self.t0 = time.time()

    def mark_end(self):
        self.t1 = time.time()

    def stop(self):
        self.run = False
        self.th.join(timeout=2)
        inside = [r for r in self.rows if self.t0 is not None and self.t0 <= r[0] <= self.t1]
        if not inside:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"], "source": "nvml"}
        reasons = sorted({n for r in inside for n, bit in self.REASONS if r[3] & bit})
        return {"sm_mhz": float(np.median([r[1] for r in inside])), "sm_max_mhz": float(max(r[2] for r in inside)),
                "reasons": reasons, "samples": len(inside), "window_s": round(self.t1 - self.t0, 4),
                "power_w_max": float(max(r[4] for r in inside)), "source": "nvml, 2 ms"}


def clock_sampler(local):
    """NVML sampler where the library loads, else nvidia-smi."""
    try:
        return NvmlClockSampler(local)
    except Exception:
        return ClockSampler(local)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled every 50 ms from before
    the warm-up on; stop() keeps the samples whose nvidia-smi timestamp falls
    inside the timed region [mark_start(), mark_end()]."""
    Q = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None
        self.t0 = self.t1 = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
        except Exception:
            self.proc = None

    def _read(self):
        import datetime
        for line in self.proc.stdout:
            r = [x.strip() for x in line.split(",")]
            try:
                ts = datetime.datetime.strptime(r[0], "%Y/%m/%d %H:%M:%S.%f").timestamp()
            except Exception:
                continue
            self.rows.append([ts] + r[1:])

    def mark_start(self):
        self.t0 = time.time()

    def mark_end(self):
        self.t1 = time.time()

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.2)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = [r for r in self.rows if len(r) >= 10]
        inside = [r for r in rows if self.t0 is not None and self.t0 - 0.025 <= r[0] <= self.t1 + 0.025]
        use = inside
        if not use:   # region shorter than the sampling period: the samples around it
            after = [r for r in rows if self.t0 is not None and r[0] >= self.t0]
            before = [r for r in rows if self.t0 is not None and r[0] < self.t0]
            use = after[:1] + before[-1:]
        if not use:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[2]) for r in use if r[2].replace(".", "").isdigit()]
        mx = [float(r[3]) for r in use if r[3].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in use for k in range(4) if r[6 + k].lower().startswith("active")})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(inside), "window_s": round(self.t1 - self.t0, 3)}


def setup_model(nx, ny, seed=0):
    from xbeach_gpu_b200.model import Model
    from xbeach_gpu_b200.scenarios import make_case
    p, zb, bnd = make_case("barred_beach", seed=seed, nx=nx, ny=ny)
    m = Model(p)
    m.set_wave_boundary(0, bnd["St"], bnd["q"], t0=0.0, tend=p.rtlength, Trep=bnd["Trep"])
    m.set_sealevel([0.0, 1e6], [0.0, 0.0], [0.0, 0.0])
    m.set_wind([0.0, 1e6], [0.0, 0.0], [0.0, 0.0])
    m.init_state(zb, 0.0, 0.0)
    return p, m, bnd


def cpu_baseline_port(nx_full, ny_full, seconds=12.0):
    """The oracle (CPU restatement, serial) on a 256 x 128 crop of the same
    barred-beach workload, run for a bounded time: cell-updates/s, 1 core."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    from xbeach_gpu_b200.scenarios import make_case
    nx, ny = 256, 128
    p, zb, bnd = make_case("barred_beach", nx=nx, ny=ny)
    o = pyoracle.Oracle(p)
    o.set_wave_boundary(0, bnd["St"], bnd["q"], t0=0.0, tend=p.rtlength, Trep=bnd["Trep"])
    o.set_sealevel([0.0, 1e6], [0.0, 0.0], [0.0, 0.0])
    o.set_wind([0.0, 1e6], [0.0, 0.0], [0.0, 0.0])
    o.init_state(zb, 0.0, 0.0)
    o.advance(2)
    t0 = time.perf_counter()
    n = 0
    while time.perf_counter() - t0 < seconds:
        o.advance(2)
        n += 2
    el = time.perf_counter() - t0
    return {"value": nx * ny * n / el, "unit": "cell-updates/s", "cores": 1, "kind": "port",
            "sample": f"oracle restatement, serial, barred beach crop {nx}x{ny} ntheta={p.ntheta}, "
                      f"{n} coupled steps in {el:.1f} s"}


def _ref_worker(job):
    """One host core: the reference's CPU code on a barred-beach crop, `steps`
    steps after `warmup`, stopping early after `limit` seconds; returns
    (timed steps, seconds, cells)."""
    import numpy as np
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    sys.path.insert(0, ROOT)
    import pyoracle
    from xbeach_gpu_b200.abi import FIELD_NAMES
    from xbeach_gpu_b200.scenarios import make_case
    nx, ny, seed, steps, warmup, limit, presteps = job
    p, zb, bnd = make_case("barred_beach", nx=nx, ny=ny, seed=seed)
    o = pyoracle.Oracle(p)   # a physically consistent starting state
    o.set_wave_boundary(0, bnd["St"], bnd["q"], t0=0.0, tend=p.rtlength, Trep=bnd["Trep"])
    o.set_sealevel([0.0, 1e6], [0.0, 0.0], [0.0, 0.0])
    o.set_wind([0.0, 1e6], [0.0, 0.0], [0.0, 0.0])
    o.init_state(zb, 0.0, 0.0)
    o.advance(presteps)
    r = pyoracle.RefEmu(p)
    for n in FIELD_NAMES:
        r.set(n, o.get(n))
    t, dt, _, _, _ = o.time()
    del o
    nb = int(t // p.dtbc)
    St = bnd["St"][nb].astype(np.float32)
    q0, q1 = bnd["q"][nb].astype(np.float32), bnd["q"][nb + 1].astype(np.float32)
    trep = np.float32(bnd["Trep"])
    del bnd
    per = []
    for k in range(warmup + steps):
        r.step_inputs(dt, t + k * dt, trep, St, q0, q1, 0.5, 1.0, 0.0, 0.0, 0.0, 0.0)
        t0 = time.perf_counter()
        for call in ("wave_step", "flow_boundary", "flow_step", "sediment_step"):
            r.call(call)
        per.append(time.perf_counter() - t0)
        if sum(per) > limit:
            break
    timed = per[min(warmup, len(per) - 1):]
    return len(timed), float(np.sum(timed)), nx * ny


def reference_replicas(cores, avail_bytes, nx, ny):
    """How many whole-domain replicas of the reference's serial CPU code to
    run: one per core, as many as the host memory holds at about 6 GB per
    2048 x 1024 replica (the boundary series and two model states), and at
    most 16 -- a whole-domain step takes tens of seconds and the replicas
    share the host's memory bandwidth, so more would only stretch the run
    past a few minutes."""
    n = max(1, cores)
    if avail_bytes is not None:
        n = min(n, int(avail_bytes // (6e9 * max(1.0, nx * ny / 2.1e6))))
    return max(1, min(n, 16))


def run_reference(args, rank, world):
    """--impl reference: the reference's own CPU code (wave_CPU.cpp and its flow
    and sediment kernels run on the CPU, oracle/_ref) on the host cores: the
    reference code is serial, so each core runs an independent replica of the
    whole benchmarked domain (the barred beach at --nx x --ny, 18 bins; as
    many replicas as cores, at most 16 and bounded by the host memory at about
    6 GB each), each timing whole steps (at least one) until a 60 s cap, and
    the value is their summed cell-updates/s."""
    if rank != 0:
        return None
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import multiprocessing as mp
    import pyoracle
    if not pyoracle.ref_available():
        return {"impl": "reference", "unavailable": "oracle/_ref/libxbg_ref.so not built (needs the reference checkout at build time)"}
    try:
        cores = len(os.sched_getaffinity(0))
    except Exception:
        cores = os.cpu_count() or 1
    nx, ny = args.nx, args.ny
    try:
        avail = os.sysconf("SC_AVPHYS_PAGES") * os.sysconf("SC_PAGE_SIZE")
    except (ValueError, OSError):
        avail = None
    cores = reference_replicas(cores, avail, nx, ny)
    jobs = [(nx, ny, k, max(1, args.steps), 0, 60.0, 1) for k in range(cores)]
    with mp.get_context("spawn").Pool(cores) as pool:
        res = pool.map(_ref_worker, jobs)
    v = float(sum(n * c / max(s, 1e-9) for n, s, c in res))
    steps = int(min(n for n, _, _ in res))
    ms = 1e3 * float(np.mean([s / max(n, 1) for n, s, _ in res]))
    sample = (f"reference wave_CPU.cpp + reference flow/sediment kernels on the CPU, one serial replica of the "
              f"whole {nx}x{ny} ntheta=18 barred beach per core ({cores} cores), >= {steps} timed steps each "
              f"(60 s cap per replica)")
    return {"metric": "coupled cell-updates/s", "value": v, "unit": "cell-updates/s", "impl": "reference",
            "n_gpus": args.gpus, "steps": steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded barred beach)",
            "config": {"workload": f"barred_beach {args.nx}x{args.ny} ntheta=18 (large single domain)",
                       "nx": nx, "ny": ny, "ntheta": 18, "cells": nx * ny,
                       "parallelism": f"{cores} serial replicas, one per core"},
            "cpu_baseline": {"value": v, "unit": "cell-updates/s", "cores": cores, "kind": "reference",
                             "sample": sample},
            "e2e": {"value": v, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def run_ensemble(args, rank, world, local):
    """The batched ensemble: args.scenarios ragged scenarios (nx 128..1024,
    ny 64..512, 12 bins) advanced together, one launch per kernel of the step
    for all of them; value = sum of cells x steps / CUDA-event time."""
    import torch
    from xbeach_gpu_b200.model import Batch
    from xbeach_gpu_b200.scenarios import iter_ensemble, make_ensemble
    torch.cuda.set_device(local)
    params = [p for p, _, _ in iter_ensemble(args.scenarios, seed=rank, boundary=False)]
    b = Batch(params)
    cells = 0
    for s, (p, zb, bnd) in enumerate(iter_ensemble(args.scenarios, seed=rank)):
        m = b.scenario(s)
        m.set_wave_boundary(0, bnd["St"], bnd["q"], t0=0.0, tend=p.rtlength, Trep=bnd["Trep"])
        m.set_sealevel([0.0, 1e6], [0.0, 0.0], [0.0, 0.0])
        m.set_wind([0.0, 1e6], [0.0, 0.0], [0.0, 0.0])
        m.init_state(zb, 0.0, 0.0)
        cells += p.nx * p.ny
    tuned = None
    if not args.no_autotune:
        from xbeach_gpu_b200.autotune import tune
        tuned = tune(b, reps=2)
    stream = torch.cuda.ExternalStream(b.stream())
    W, K = max(3, args.warmup), args.steps
    sampler = clock_sampler(local)
    sampler.start()
    b.advance(W)
    b.sync()
    l0 = b.launches()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    sampler.mark_start()
    ev0.record(stream)
    b.advance(K)
    ev1.record(stream)
    ev1.synchronize()
    sampler.mark_end()
    clocks = sampler.stop()
    ms = ev0.elapsed_time(ev1)
    st = b.status()
    if (st["status"] != 0).any():
        raise RuntimeError("a scenario reported an error")
    launches = b.launches() - l0
    prof = {}
    for _ in range(3):
        for name, t in b.profile_step():
            prof.setdefault(name, []).append(t)
    kern = {k: float(np.mean(v)) for k, v in prof.items()}
    nt = params[0].ntheta
    wrows = sum(p.nx * (p.ny - 2) for p in params)
    peak, peak_kind = peaks()
    dom = max(kern, key=kern.get)
    roof = None
    if dom in ("k_wave_fast", "k_wave_tma"):
        achieved = 4 * (4 * nt + 16) * wrows / (kern[dom] / 1e3) / 1e9
        roof = {"kernel": dom, "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_kind": peak_kind, "traffic": None,
                "algorithmic_bytes_per_cell": 4 * (4 * nt + 16), "ms_per_launch": kern[dom]}
    value = cells * K / (ms / 1e3)
    step_gbs = B_ALGO(nt) * cells * K / (ms / 1e3) / 1e9
    out = {
        "metric": "coupled cell-updates/s", "value": value, "unit": "cell-updates/s", "n_gpus": world,
        "steps": K, "warmup": W, "ms_per_step": ms / K, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded ragged ensemble)",
        "config": {"workload": f"ragged ensemble of {args.scenarios} scenarios, nx 128..1024, ny 64..512, "
                               f"ntheta={nt}, one batched launch per kernel", "scenarios": args.scenarios,
                   "cells": cells, "parallelism": f"replicas x{world}",
                   "l2": "state ~20 GB per GPU, larger than the 126 MB L2 (no flush needed)"},
        "roofline": roof,
        "roofline_step": {"bound": "hbm", "achieved": step_gbs, "peak": peak, "unit": "GB/s",
                          "frac": step_gbs / peak, "algorithmic_bytes_per_cell_update": B_ALGO(nt),
                          "peak_kind": peak_kind},
        "kernels_ms": kern, "gpu_launches": int(launches), "clocks": clocks,
        "sim_time_s": [float(st["t"].min()), float(st["t"].max())],
        "autotuned_blocks": {str(k): v for k, v in (tuned or {}).items()},
    }
    b.close()
    return out


def run_surrogate(args, rank, world, local):
    """The wave surrogate: train on snapshot pairs of plain runs, infer on a
    1024 x 512 domain, and run the coupled step with the wave sub-steps from
    the surrogate (judged by the plain solver every 50 steps, 2% H bar)
    beside the plain step on the same held-out beach."""
    import torch
    from xbeach_gpu_b200 import surrogate_train as st
    from xbeach_gpu_b200.surrogate import UNet
    from xbeach_gpu_b200.surrogate_couple import SurrogateRun
    torch.cuda.set_device(local)
    t0 = time.perf_counter()
    train_d = st.collect(nx=512, ny=256, seeds=(0, 1, 2), Hs_list=(1.5, 2.5, 3.5), warm=300, every=15, count=12, k=10)
    test_d = st.collect(nx=512, ny=256, seeds=(7,), Hs_list=(2.0,), warm=300, every=15, count=6, k=10)
    t_collect = time.perf_counter() - t0
    norm = st.Normalizer(train_d)
    net = UNet(seed=0, base=args.surrogate_base)
    steps = max(200, args.steps * 3)
    t0 = time.perf_counter()
    hist = st.train(net, train_d, norm, steps=steps, batch=16, crop=128, lr=5e-4, log_every=max(1, steps // 6))
    t_train = time.perf_counter() - t0
    res, _ = st.evaluate(net, norm, test_d)
    # useful FLOPs of one forward pass per pixel (3x3 convolutions, by level)
    scale = {"e1a": 1, "e1b": 1, "d1a": 1, "d1b": 1, "head": 1, "e2a": 4, "e2b": 4, "d2a": 4, "d2b": 4,
             "e3a": 16, "e3b": 16, "d3a": 16, "d3b": 16, "e4a": 64, "e4b": 64}
    fwd_per_px = sum(2.0 * 9 * l.cin * l.cout / scale[n] for n, l in net.L.items())
    xb, yb = next(st.batches(train_d, norm, 16, 128, np.random.default_rng(3)))
    for _ in range(3):
        net.train_step(xb, yb, 16, 128, 128)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(10):
        net.train_step(xb, yb, 16, 128, 128)
    e1.record(); e1.synchronize()
    train_ms = e0.elapsed_time(e1) / 10
    train_tflops = 3 * fwd_per_px * 16 * 128 * 128 / (train_ms / 1e3) / 1e12
    nyi, nxi = 512, 1024
    xi = torch.zeros(nyi * nxi, xb.shape[1], dtype=torch.bfloat16, device="cuda")
    for _ in range(3):
        net.forward(xi, 1, nyi, nxi)
    e0.record()
    for _ in range(10):
        net.forward(xi, 1, nyi, nxi)
    e1.record(); e1.synchronize()
    infer_ms = e0.elapsed_time(e1) / 10
    infer_tflops = fwd_per_px * nyi * nxi / (infer_ms / 1e3) / 1e12
    net.check()
    # coupled: plain vs surrogate-assisted on a held-out 1024 x 512 beach
    nsteps = 400

    def timed(fn):   # CUDA events on the default stream around host-driven steps
        torch.cuda.synchronize()
        e0.record()
        fn()
        e1.record(); e1.synchronize()
        return e0.elapsed_time(e1) / 1e3

    a, Tp = st.beach_model(2.2, seed=9, nx=1024, ny=512, warm=300)
    b, _ = st.beach_model(2.2, seed=9, nx=1024, ny=512, warm=300)
    c, _ = st.beach_model(2.2, seed=9, nx=1024, ny=512, warm=300)

    def plain():
        a.advance(nsteps); a.sync()
    t_plain = timed(plain)
    run = SurrogateRun(b, net, norm, Hs=2.2, Tp=Tp, k=10, judge_every=50, threshold=0.02)
    t_judged = timed(lambda: run.advance(nsteps))
    free = SurrogateRun(c, net, norm, Hs=2.2, Tp=Tp, k=10, judge_every=50, threshold=float("inf"))
    t_sur = timed(lambda: free.advance(nsteps))
    final = {f: st.rel_err(b.get(f), a.get(f)) for f in ("H", "zb", "zs")}
    final_free = {f: st.rel_err(c.get(f), a.get(f)) for f in ("H", "zb", "zs")}
    peak_tc = None
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peak_tc = float(json.load(f)["bf16_tflops"])
    except Exception:
        peak_tc = 1590.0
    cells = 1024 * 512
    return {
        "metric": "coupled cell-updates/s", "value": cells * nsteps / t_sur, "unit": "cell-updates/s",
        "impl": "surrogate", "n_gpus": world, "steps": nsteps, "higher_is_better": True, "dtype": "bf16/f32",
        "data": "synthetic (plain-run snapshots of seeded barred beaches)",
        "config": {"workload": "surrogate-assisted coupled step, 1024x512 barred beach, k=10, judge every 50 "
                               "(value: judge without a bar, 80% surrogate steps)",
                   "train_crops": "16 x 128 x 128",
                   "net": f"U-Net 4 levels, {args.surrogate_base} base channels, 3x3"},
        "plain_value": cells * nsteps / t_plain,
        "speedup_vs_plain": t_plain / t_sur,
        "unjudged_final_rel_err_vs_plain": final_free,
        "judged_2pct": {"judged": run.judged, "fallback": run.fallback, "surrogate_steps": run.surrogate_steps,
                        "value": cells * nsteps / t_judged, "final_rel_err_vs_plain": final},
        "heldout_rel_err": res,
        "train": {"steps": steps, "seconds": t_train, "loss": hist, "ms_per_step": train_ms,
                  "achieved_tflops": train_tflops, "peak_tflops": peak_tc, "frac": train_tflops / peak_tc,
                  "bound": "tensor"},
        "infer_1024x512": {"ms": infer_ms, "achieved_tflops": infer_tflops, "frac": infer_tflops / peak_tc},
        "collect_s": t_collect,
    }


def run_storm(args, local):
    """The surrogate-assisted storm ensemble: n scenarios (nx 256..1024, ny
    128..512, 12 bins, morfac 10, the 6 h storm from storm time 2 h) stepped
    plain and surrogate-assisted (network trained here on snapshots of other
    storm scenarios, then two push-forward rounds; judge every 50 steps; 2 %
    bar, and without a bar) from
    the same state; cell-updates/s of each, final H and zb against the plain
    run, fallback rate, inference tensor throughput and the Amdahl bound of
    replacing the wave sub-step (the wave kernels' share of a plain step)."""
    import torch
    from xbeach_gpu_b200 import surrogate_train as st
    from xbeach_gpu_b200.scenarios import iter_storm_ensemble
    from xbeach_gpu_b200.surrogate import UNet
    from xbeach_gpu_b200.surrogate_couple import BatchSurrogateRun
    torch.cuda.set_device(local)
    t_all = time.perf_counter()
    train_sc = list(iter_storm_ensemble(16, seed=100, nx_range=(128, 256), ny_range=(96, 160)))
    data = st.collect_batch(train_sc, warm=150, every=12, count=16, k=10, crop=96, crops_per=4, seed=1)
    norm = st.Normalizer(data)
    net = UNet(seed=0, base=32)
    t0 = time.perf_counter()
    st.train(net, data, norm, steps=2000, batch=16, crop=96, lr=5e-4, log_every=500)
    # push-forward rounds against chained drift: pairs whose held wave fields
    # are the network's own prediction one link earlier on plain chains of
    # the training scenarios, trained with the plain pairs
    chain = st.collect_chain(train_sc, warm=160, k=10, links=8, crop=96, crops_per=4, seed=3)
    plain_pairs = st.chain_pairs(chain)
    pf_rounds = 2
    for r in range(pf_rounds):
        pf = st.pushforward_pairs(net, norm, chain)
        st.train(net, st.merge(data, plain_pairs, pf), norm, steps=1500, batch=16, crop=96, lr=2.5e-4, seed=r + 1,
                 log_every=500)
    t_train = time.perf_counter() - t0
    sc = list(iter_storm_ensemble(args.storm_scenarios, seed=7, rtlength=600.0))
    params = [p for p, _, _ in sc]
    cells = sum(p.nx * p.ny for p in params)
    K, warm = args.storm_steps, 200   # the wave field established over the domains before the comparison
    storm = lambda s, t: sc[s][2]["storm"](t)   # noqa: E731
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    out = {"scenarios": len(sc), "cells": cells, "steps": K, "k": 10, "judge_every": 50, "train_s": t_train,
           "train_crops": int(data["x"].shape[0]), "pushforward_rounds": pf_rounds,
           "pushforward_pairs": int(pf["x"].shape[0])}
    finals = {}
    for mode in ("plain", "2pct", "nobar"):
        b = st.storm_batch(sc, warm)
        if mode == "plain":   # (the default persistent grids in all three runs)
            prof = {}
            for _ in range(2):
                for name, t in b.profile_step():
                    prof.setdefault(name, []).append(t)
            kern = {k: float(np.mean(v)) for k, v in prof.items()}
            wave = sum(v for k, v in kern.items() if k in ("k_disp", "k_wave_tma", "k_wave_fast", "k_wave_force",
                                                               "k_wavebnd"))
            out["wave_share"] = wave / sum(kern.values())
            out["amdahl_bound"] = 1.0 / (1.0 - out["wave_share"])
            b.sync()
            stream = torch.cuda.ExternalStream(b.stream())
            e0.record(stream)
            b.advance(K)
            e1.record(stream)
            e1.synchronize()
        else:
            b.advance(2)   # the plain run's two profiled steps: all three start from the same step
            thr = 0.02 if mode == "2pct" else float("inf")
            run = BatchSurrogateRun(b, params, net, norm, storm, k=10, judge_every=50, threshold=thr, hp=64, wp=128)
            torch.cuda.synchronize()
            e0.record()
            run.advance(K)
            torch.cuda.synchronize()
            e1.record()
            e1.synchronize()
        ms = e0.elapsed_time(e1)
        stt = b.status()
        if (stt["status"] != 0).any():
            raise RuntimeError(f"storm ensemble ({mode}): a scenario reported an error")
        finals[mode] = [{f: b.scenario(s).get(f).astype(np.float64) for f in ("H", "zb")} for s in range(len(sc))]
        out[f"{mode}_value"] = cells * K / (ms / 1e3)
        if mode != "plain":
            out[f"{mode}_fallback_rate"] = float(run.fallback.mean())
            out[f"{mode}_judged_median"] = [[j, float(np.median(e[e >= 0])) if (e >= 0).any() else None]
                                            for j, e in run.judged]
        b.close()
    for mode in ("2pct", "nobar"):
        out[f"{mode}_speedup_vs_plain"] = out[f"{mode}_value"] / out["plain_value"]
        for f in ("H", "zb"):
            errs = [np.linalg.norm(a[f] - r[f]) / max(np.linalg.norm(r[f]), 1e-30)
                    for a, r in zip(finals[mode], finals["plain"])]
            out[f"{mode}_final_rel_err_{f}"] = {"median": float(np.median(errs)), "max": float(np.max(errs))}
    # inference on one 1024 x 512 domain: tensor throughput of the network
    fwd_px = sum(2.0 * 9 * l.cin * l.cout / {"e1": 1, "d1": 1, "he": 1, "e2": 4, "d2": 4, "e3": 16, "d3": 16,
                                               "e4": 64}[n[:2]] for n, l in net.L.items())
    xi = torch.zeros(512 * 1024, 16, dtype=torch.bfloat16, device="cuda")
    for _ in range(3):
        net.forward(xi, 1, 512, 1024)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(10):
        net.forward(xi, 1, 512, 1024)
    e1.record()
    e1.synchronize()
    infer_ms = e0.elapsed_time(e1) / 10
    tflops = fwd_px * 512 * 1024 / (infer_ms / 1e3) / 1e12
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peak_tc, kind = float(json.load(f)["bf16_tflops"]), "measured"
    except Exception:
        peak_tc, kind = 1590.0, "fallback"
    out["infer_1024x512"] = {"ms": infer_ms, "achieved_tflops": tflops, "peak_tflops": peak_tc, "peak_kind": kind,
                             "frac": tflops / peak_tc, "bound": "tensor"}
    net.check()
    out["wall_s"] = time.perf_counter() - t_all
    return out


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist_
        dist = dist_
        import torch
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    if args.impl == "reference":
        out = run_reference(args, rank, world)
        if out is not None:
            print(json.dumps(out), flush=True)
        if dist:
            dist.destroy_process_group()
        return
    import torch
    torch.cuda.set_device(local)
    if args.workload == "surrogate":
        out = run_surrogate(args, rank, world, local) if rank == 0 else None
        if out is not None:
            print(json.dumps(out), flush=True)
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return
    if args.workload == "storm":
        out = run_storm(args, local) if rank == 0 else None
        if out is not None:
            print(json.dumps({"metric": "coupled cell-updates/s", "value": out["2pct_value"],
                              "unit": "cell-updates/s", "impl": "surrogate-ensemble", "n_gpus": 1,
                              "higher_is_better": True, "storm": out}), flush=True)
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return
    if args.workload == "ensemble":
        out = run_ensemble(args, rank, world, local)
        if dist:
            (msx,), (cells,) = over_ranks(dist, [out["ms_per_step"]], [out["config"]["cells"]], "cuda")
            out["ms_per_step"] = msx
            out["value"] = cells / (msx / 1e3)
        if rank == 0:
            print(json.dumps(out), flush=True)
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return
    from xbeach_gpu_b200.abi import XBG_FLAG_ENDED, XBG_FLAG_OUTPUT_DUE
    p, m, bnd = setup_model(args.nx, args.ny, seed=rank)
    C = p.nx * p.ny
    stream = torch.cuda.ExternalStream(m.stream())
    W = max(3, args.warmup)
    K = args.steps
    sampler = clock_sampler(local)
    sampler.start()
    m.advance(W)
    m.sync()
    _, _, nstep0, flags0, rc0 = m.time()
    if rc0 != 0 or nstep0 != W or flags0 & (XBG_FLAG_OUTPUT_DUE | XBG_FLAG_ENDED):
        raise RuntimeError(f"warm-up did not run W steps (status {rc0}, steps {nstep0}, flags {flags0})")
    launches0 = m.launches()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    sampler.mark_start()
    ev0.record(stream)
    m.advance(K)
    ev1.record(stream)
    ev1.synchronize()
    sampler.mark_end()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clocks = sampler.stop()
    ms = ev0.elapsed_time(ev1)
    t_end, dt_end, nstep, flags, rc = m.time()
    if rc != 0:
        raise RuntimeError(f"device status {rc} after the timed steps")
    # every timed replay ran a whole step: the device clock advanced by K steps
    # and no end-of-run or output stop was reached inside the region
    if nstep != nstep0 + K or flags & (XBG_FLAG_OUTPUT_DUE | XBG_FLAG_ENDED):
        raise RuntimeError(f"timed region ran {nstep - nstep0} of {K} steps (flags {flags})")
    launches = m.launches() - launches0
    # per-kernel times of full steps (events between launches), for the roofline
    prof = {}
    for _ in range(5):
        for name, t in m.profile_step():
            prof.setdefault(name, []).append(t)
    kern = {k: float(np.mean(v)) for k, v in prof.items()}
    # end to end through the C ABI with host buffers: every step uploads the
    # boundary records around its time (St and qbnd) from pinned host memory
    # and copies its clock (time, dt, step count, status) back into pinned
    # host memory (xbg_get_time_async); the host decodes step k's clock while
    # step k+1 runs, and chooses step k+2's records from it (four records
    # from the one at that time on bracket the two steps' times), so host and
    # device work overlap instead of alternating
    from xbeach_gpu_b200.abi import XBG_CLOCK_BYTES
    nyt = p.ny * p.ntheta
    NR = 4
    recs = [torch.empty((NR, nyt), dtype=torch.float32, pin_memory=True) for _ in range(2)]
    qrec = [torch.empty((NR, 4 * p.ny), dtype=torch.float32, pin_memory=True) for _ in range(2)]
    clkb = [torch.empty(XBG_CLOCK_BYTES, dtype=torch.uint8, pin_memory=True) for _ in range(2)]
    evs = [torch.cuda.Event() for _ in range(2)]
    Ke = max(10, K // 4)
    t_known, _, n_e0, _, _ = m.time()
    nrec = bnd["St"].shape[0]
    rc = 0
    t0 = time.perf_counter()
    for k in range(Ke):
        b = k % 2
        if k >= 2:   # step k-2 has finished: its clock is in clkb[b], its buffers are free
            evs[b].synchronize()
            t_known, _, _, _, rc = m.time_decode(clkb[b].data_ptr())
            if rc != 0:
                break
        nb = min(int(t_known // p.dtbc), nrec - NR)
        recs[b].numpy()[:] = bnd["St"][nb:nb + NR].reshape(NR, -1)
        qrec[b].numpy()[:] = bnd["q"][nb:nb + NR].reshape(NR, -1)
        m.put_wave_records(0, nb, recs[b].numpy(), qrec[b].numpy())
        m.step()
        m.time_async(clkb[b].data_ptr())
        evs[b].record(stream)
    for k in range(max(0, Ke - 2), Ke):   # the last two steps' clocks
        evs[k % 2].synchronize()
        _, _, n_e, _, rck = m.time_decode(clkb[k % 2].data_ptr())
        rc = rc or rck
    e2e_s = time.perf_counter() - t0
    if rc != 0 or n_e != n_e0 + Ke:
        raise RuntimeError(f"end-to-end steps: status {rc}, {n_e - n_e0} of {Ke} steps")
    h2d = recs[0].numel() * 4 + qrec[0].numel() * 4
    # the clocks over a longer run of the same replays (>= 250 ms of device
    # work), so the clock record does not rest on the few samples a short
    # timed region allows; the timed region's own samples stay in "clocks"
    soak = clock_sampler(local)
    soak.start()
    n_soak = max(1, int(np.ceil(250.0 / max(ms / K, 1e-3))))
    torch.cuda.synchronize()
    soak.mark_start()
    m.advance(n_soak)
    m.sync()
    soak.mark_end()
    clocks_soak = soak.stop()
    clocks_soak["steps"] = n_soak
    d2h = XBG_CLOCK_BYTES   # the device clock copied back by xbg_get_time_async
    # max over ranks
    if dist:
        (ms, e2e_s), _ = over_ranks(dist, [ms, e2e_s], [C], "cuda")
    value = C * K * world / (ms / 1e3)
    e2e = C * Ke * world / e2e_s
    peak, peak_kind = peaks()
    # dominant kernel: the fused wave-action kernel
    dom = max(kern, key=kern.get)
    nt = p.ntheta
    wave_rows = ("k_wave_fast", "k_wave_tma")
    algo_dom = 4 * (4 * nt + 16) if dom in wave_rows else None
    rows = p.ny - 2 if dom in wave_rows else p.ny
    roof = None
    if algo_dom:
        achieved = algo_dom * p.nx * rows / (kern[dom] / 1e3) / 1e9
        roof = {"kernel": dom, "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_kind": peak_kind,
                "traffic": NCU_TRAFFIC.get((dom, p.nx, p.ny, nt)),
                "algorithmic_bytes_per_cell": algo_dom, "ms_per_launch": kern[dom]}
    step_gbs = B_ALGO(nt) * C * K / (ms / 1e3) / 1e9
    out = {
        "metric": "coupled cell-updates/s", "value": value, "unit": "cell-updates/s", "n_gpus": world,
        "steps": K, "warmup": W, "ms_per_step": ms / K, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded barred beach, JONSWAP-shaped groups)",
        "config": {"workload": f"barred_beach {p.nx}x{p.ny} ntheta={nt} (large single domain)",
                   "nx": p.nx, "ny": p.ny, "ntheta": nt, "cells": C, "parallelism": f"replicas x{world}",
                   "l2": "state ~1.2 GB per GPU, larger than the 126 MB L2 (no flush needed)",
                   "sim_time_s": t_end},
        "roofline": roof,
        "roofline_step": {"bound": "hbm", "achieved": step_gbs, "peak": peak, "unit": "GB/s",
                          "frac": step_gbs / peak, "algorithmic_bytes_per_cell_update": B_ALGO(nt),
                          "peak_kind": peak_kind},
        "kernels_ms": kern,
        "e2e": {"value": e2e, "unit": "cell-updates/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "gpu_launches": int(launches),
        "clocks": clocks,
        "clocks_soak": clocks_soak,
    }
    if rank == 0 and not args.no_cpu_baseline:
        try:
            out["cpu_baseline"] = cpu_baseline_port(p.nx, p.ny)
        except Exception as e:  # the baseline is reported, never required
            out["cpu_baseline"] = {"unavailable": str(e)}
    m.close()
    if world == 1 and not args.no_extras:
        # the batched half of the metric, measured in the same run: the plain
        # ragged ensemble (256 scenarios) and the surrogate-assisted storm
        # ensemble (512 scenarios) beside its own plain run
        try:
            ea = argparse.Namespace(scenarios=256, steps=min(K, 20), warmup=3, no_autotune=False)
            e = run_ensemble(ea, 0, 1, local)
            out["ensemble"] = {k: e[k] for k in ("value", "ms_per_step", "steps", "roofline", "roofline_step",
                                                  "gpu_launches", "clocks", "autotuned_blocks")}
            out["ensemble"]["workload"] = e["config"]["workload"]
            out["ensemble"]["cells"] = e["config"]["cells"]
        except Exception as ex:
            out["ensemble"] = {"unavailable": f"{type(ex).__name__}: {ex}"}
        try:
            out["storm_ensemble"] = run_storm(args, local)
        except Exception as ex:
            out["storm_ensemble"] = {"unavailable": f"{type(ex).__name__}: {ex}"}
    if rank == 0:
        print(json.dumps(out), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
