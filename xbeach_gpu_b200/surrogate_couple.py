"""Surrogate-assisted stepping of one domain, judged by the plain wave solver.

The coupled step runs as usual except for the wave action sub-steps.  In a
surrogate segment of k steps the network predicts the wave fields E, H, D,
DR, Fx, Fy k steps ahead from the current state; for steps j = 1..k of the
segment the forcing is f(t) + (j/k) (prediction - f(t)) (xbg_set_wave_forcing
in place of the wave step), and at the end the wave action and roller
energy are rescaled per cell to the predicted E and DR so the plain solver can
take over from a consistent state.  Every `judge_every` steps a judge segment
runs k full plain steps (wave solver included) from the current state and
compares their H with the network's prediction for the same k steps; when the
relative L2 error exceeds `threshold` the run falls back to the plain method
for good.  Flow, sediment, dt and boundaries are the plain kernels throughout.

The k forced steps of a segment run as one CUDA graph (xbg_forcing_steps).
The network's kernels run on the default stream and the model's on its own;
CUDA events order the two (the network reads the model's state after the
model's last step, the forced steps read the prediction after the network),
so a segment needs no host synchronisation.
"""
import numpy as np

from .abi import XBG_WAVE_FALLBACK, XBG_WAVE_FORCED, XBG_WAVE_PLAIN
from .surrogate import IN_CH, OUT_CH, _ok, _p, lib
from .surrogate_train import IN_FIELDS, OUT_FIELDS


class SurrogateRun:
    def __init__(self, model, net, norm, Hs, Tp, k=10, judge_every=50, threshold=0.02):
        import torch
        self.m, self.net, self.norm = model, net, norm
        self.nx, self.ny = model.p.nx, model.p.ny
        self.P = P = self.nx * self.ny
        self.k, self.judge_every, self.threshold = k, judge_every, threshold
        dev = "cuda"
        f32 = torch.float32
        self.planes = [torch.full((P,), float(Hs), dtype=f32, device=dev),
                       torch.full((P,), float(Tp), dtype=f32, device=dev)]
        self.f0 = torch.empty(OUT_CH, P, dtype=f32, device=dev)     # forcing at the segment start
        self.f1 = torch.empty(OUT_CH, P, dtype=f32, device=dev)     # predicted forcing k steps on
        self.x = torch.empty(P, IN_CH, dtype=torch.bfloat16, device=dev)
        wave = [model.device_ptr(f)[0] for f in OUT_FIELDS]
        enc = [model.device_ptr(f)[0] for f in IN_FIELDS] + [t.data_ptr() for t in self.planes] + wave
        enc += [0] * (IN_CH - len(enc))
        self.enc = torch.tensor(enc, dtype=torch.int64, device=dev)
        self.wave = torch.tensor(wave, dtype=torch.int64, device=dev)
        self.f0p = torch.tensor([self.f0[c].data_ptr() for c in range(OUT_CH)], dtype=torch.int64, device=dev)
        self.f1p = torch.tensor([self.f1[c].data_ptr() for c in range(OUT_CH)], dtype=torch.int64, device=dev)
        self.xm = torch.from_numpy(norm.xm.astype(np.float32)).to(dev)
        self.xi = torch.from_numpy((1.0 / norm.xs).astype(np.float32)).to(dev)
        self.ym = torch.from_numpy(norm.ym.astype(np.float32)).to(dev)
        self.ys = torch.from_numpy(norm.ys.astype(np.float32)).to(dev)
        self.f0_ptrs = [self.f0[c].data_ptr() for c in range(OUT_CH)]
        self.f1_ptrs = [self.f1[c].data_ptr() for c in range(OUT_CH)]
        self._ms = torch.cuda.ExternalStream(model.stream())
        self._ev_m = torch.cuda.Event()
        self._ev_n = torch.cuda.Event()
        self.fallback = False
        self.steps = 0
        self.judged = []          # (step, relative H error of the prediction)
        self.surrogate_steps = 0

    def _nn_after_model(self):
        """The default stream (network kernels) waits for the model's stream."""
        import torch
        self._ev_m.record(self._ms)
        torch.cuda.default_stream().wait_event(self._ev_m)

    def _model_after_nn(self):
        """The model's stream waits for the default stream."""
        import torch
        self._ev_n.record(torch.cuda.default_stream())
        self._ms.wait_event(self._ev_n)

    def _predict(self):
        """f1 <- the network's wave fields k steps after the model's state
        (enqueued on the default stream after the model's work)."""
        L = lib()
        self._nn_after_model()
        _ok(L.xbg_nn_encode(_p(self.enc), IN_CH, _p(self.xm), _p(self.xi), _p(self.x), self.P, None), "encode")
        out = self.net.forward(self.x, 1, self.ny, self.nx)
        _ok(L.xbg_nn_decode(_p(out), out.shape[1], _p(self.wave), _p(self.ym), _p(self.ys), _p(self.f1p), OUT_CH,
                            self.P, None), "decode")

    def _surrogate_segment(self):
        self._predict()
        _ok(lib().xbg_nn_copy_planes(_p(self.wave), _p(self.f0p), OUT_CH, self.P, None), "copy planes")
        self._model_after_nn()
        self.m.forcing_steps(self.f0_ptrs, self.f1_ptrs, self.k)
        self.surrogate_steps += self.k

    def _judge_segment(self):
        self._predict()
        self._model_after_nn()     # the plain steps change the fields the network read
        self.m.advance(self.k)
        H = self.m.get("H").astype(np.float64)
        Hp = self.f1[OUT_FIELDS.index("H")].double().cpu().numpy()
        err = float(np.linalg.norm(Hp - H) / max(np.linalg.norm(H), 1e-30))
        self.judged.append((self.steps, err))
        if err > self.threshold:
            self.fallback = True

    def advance(self, nsteps):
        """nsteps coupled steps (rounded up to whole segments of k)."""
        done = 0
        while done < nsteps:
            if self.fallback:
                self.m.advance(nsteps - done)
                self.steps += nsteps - done
                break
            if self.steps % self.judge_every == 0:
                self._judge_segment()
            else:
                self._surrogate_segment()
            self.steps += self.k
            done += self.k
        self.m.sync()


class BatchSurrogateRun:
    """Surrogate-assisted stepping of a batch of scenarios (the ensemble
    form): every scenario of a Batch steps with the batched kernels; its wave
    sub-steps come from the network while it passes its judges and from the
    plain wave solver once it has failed one.

    A cycle of `judge_every` steps starts with a judge segment: the network
    predicts the wave fields k steps ahead for every scenario still on the
    surrogate, the whole batch takes k plain steps (wave solver included),
    and each scenario's prediction is compared with its plain H (relative L2,
    on the device, xbg_batch_rel_err); a scenario above `threshold` falls
    back to the plain method for good (XBG_WAVE_FALLBACK, flagged in
    xbg_batch_status).  The rest of the cycle are surrogate segments: one
    prediction per scenario, then k batched steps in which the surrogate
    scenarios take their wave sub-step from the forcing f0 + (j/k)(f1 - f0)
    and the fallen-back ones run the wave solver (xbg_batch_forced_segment,
    one CUDA graph).

    Inference runs on padded batches: scenarios are grouped by their size
    rounded up to (hp, wp) cells and each group (at most `max_images` per
    forward) is encoded into one [B, Hp, Wp, C] tensor (xbg_nn_encode_batch,
    padding repeats the last row / column) and decoded back into each
    scenario's forcing planes (xbg_nn_decode_batch, which also keeps the
    starting fields as f0).  storm(s, t) gives scenario s's Hm0 and Tp at
    model time t (the network's two constant input planes)."""

    def __init__(self, batch, params, net, norm, storm, k=10, judge_every=50, threshold=0.02, hp=64, wp=128,
                 max_images=48, recorder=None):
        import torch
        from .surrogate import _bind_ops
        from .surrogate_train import IN_FIELDS, OUT_FIELDS
        _bind_ops(lib())
        self.b, self.net, self.norm, self.storm = batch, net, norm, storm
        self.n = len(params)
        self.k, self.judge_every, self.threshold = k, judge_every, threshold
        dev = "cuda"
        f32 = torch.float32
        self.dims = [(p.nx, p.ny) for p in params]
        self.f0 = [torch.empty(OUT_CH, p.nx * p.ny, dtype=f32, device=dev) for p in params]
        self.f1 = [torch.empty(OUT_CH, p.nx * p.ny, dtype=f32, device=dev) for p in params]
        for s in range(self.n):
            batch.set_forcing(s, [self.f0[s][c].data_ptr() for c in range(OUT_CH)],
                              [self.f1[s][c].data_ptr() for c in range(OUT_CH)])
        self.xm = torch.from_numpy(norm.xm.astype(np.float32)).to(dev)
        self.xi = torch.from_numpy((1.0 / norm.xs).astype(np.float32)).to(dev)
        self.ym = torch.from_numpy(norm.ym.astype(np.float32)).to(dev)
        self.ys = torch.from_numpy(norm.ys.astype(np.float32)).to(dev)
        # groups of scenarios with one padded size
        groups = {}
        for s, (nx, ny) in enumerate(self.dims):
            key = ((ny + hp - 1) // hp * hp, (nx + wp - 1) // wp * wp)
            groups.setdefault(key, []).append(s)
        self.chunks = []
        for (Hp, Wp), ss in sorted(groups.items()):
            for i in range(0, len(ss), max_images):
                self.chunks.append(self._chunk(batch, ss[i:i + max_images], Hp, Wp, IN_FIELDS, OUT_FIELDS))
        self._ms = torch.cuda.ExternalStream(batch.stream())
        self._ev_m = torch.cuda.Event()
        self._ev_n = torch.cuda.Event()
        self.mode = [XBG_WAVE_PLAIN] * self.n
        self.fallback = np.zeros(self.n, bool)
        self.steps = 0
        self.judged = []          # (step, per-scenario relative H errors; -1 for fallen-back scenarios)
        self.surrogate_cell_steps = 0
        self.recorder = recorder  # before(t) / after() around each judge's plain steps (training data)

    def _chunk(self, batch, ss, Hp, Wp, in_fields, out_fields):
        import torch
        dev = "cuda"
        enc, hold, dst, dst0, dims = [], [], [], [], []
        for s in ss:
            m = batch.scenario(s)
            wave = [m.device_ptr(f)[0] for f in out_fields]
            e = [m.device_ptr(f)[0] for f in in_fields] + [0, 0] + wave
            enc += e + [0] * (IN_CH - len(e))
            hold += wave
            dst += [self.f1[s][c].data_ptr() for c in range(OUT_CH)]
            dst0 += [self.f0[s][c].data_ptr() for c in range(OUT_CH)]
            dims += list(self.dims[s])
        c = dict(ss=ss, Hp=Hp, Wp=Wp, B=len(ss),
                 enc=torch.tensor(enc, dtype=torch.int64, device=dev),
                 hold=torch.tensor(hold, dtype=torch.int64, device=dev),
                 dst=torch.tensor(dst, dtype=torch.int64, device=dev),
                 dst0=torch.tensor(dst0, dtype=torch.int64, device=dev),
                 dims=torch.tensor(dims, dtype=torch.int32, device=dev),
                 cval=torch.zeros(len(ss) * IN_CH, dtype=torch.float32, device=dev),
                 x=torch.empty(len(ss) * Hp * Wp, IN_CH, dtype=torch.bfloat16, device=dev))
        c["hs_slot"] = [j * IN_CH + len(in_fields) for j in range(len(ss))]
        return c

    def _predict(self, t, keep_start):
        """f1 (and f0 when keep_start) of every scenario still on the
        surrogate, from the state at model time t."""
        import torch
        from .surrogate import _p
        L = lib()
        self._ev_m.record(self._ms)
        torch.cuda.default_stream().wait_event(self._ev_m)
        for c in self.chunks:
            if all(self.fallback[s] for s in c["ss"]):
                continue
            cv = np.zeros(c["B"] * IN_CH, np.float32)
            for j, s in enumerate(c["ss"]):
                hs, tp = self.storm(s, t)
                cv[c["hs_slot"][j]], cv[c["hs_slot"][j] + 1] = hs, tp
            c["cval"].copy_(torch.from_numpy(cv), non_blocking=False)
            _ok(L.xbg_nn_encode_batch(_p(c["enc"]), IN_CH, _p(c["dims"]), _p(c["cval"]), _p(self.xm), _p(self.xi),
                                      _p(c["x"]), c["B"], c["Hp"], c["Wp"], None), "encode batch")
            out = self.net.forward(c["x"], c["B"], c["Hp"], c["Wp"])
            _ok(L.xbg_nn_decode_batch(_p(out), out.shape[1], _p(c["hold"]), _p(self.ym), _p(self.ys), _p(c["dst"]),
                                      _p(c["dst0"]) if keep_start else None, _p(c["dims"]), OUT_CH, c["B"],
                                      c["Hp"], c["Wp"], None), "decode batch")
        self._ev_n.record(torch.cuda.default_stream())
        self._ms.wait_event(self._ev_n)

    def _set_modes(self, want):
        for s in range(self.n):
            mode = XBG_WAVE_FALLBACK if self.fallback[s] else want
            if mode != self.mode[s]:
                self.b.set_wave_mode(s, mode)
                self.mode[s] = mode

    def _time(self):
        st = self.b.status()
        return float(st["t"].min())

    def advance(self, nsteps):
        """nsteps coupled steps of every scenario (whole segments of k)."""
        from .surrogate_train import OUT_FIELDS
        done = 0
        while done < nsteps:
            t = self._time()
            active = ~self.fallback
            if self.steps % self.judge_every == 0 and active.any():
                self._predict(t, keep_start=False)
                self._set_modes(XBG_WAVE_PLAIN)
                if self.recorder:
                    self.recorder.before(t)
                self.b.advance(self.k)
                if self.recorder:
                    self.recorder.after()
                ih = OUT_FIELDS.index("H")
                preds = [self.f1[s][ih].data_ptr() if active[s] else None for s in range(self.n)]
                err = self.b.rel_err("H", preds)
                self.judged.append((self.steps, err.copy()))
                newly = active & (err > self.threshold)
                self.fallback |= newly
            else:
                if active.any():
                    self._predict(t, keep_start=True)
                self._set_modes(XBG_WAVE_FORCED)
                self.b.forced_segment(self.k)
                self.surrogate_cell_steps += self.k * sum(nx * ny for (nx, ny), a in zip(self.dims, active) if a)
            self.steps += self.k
            done += self.k
        self.b.sync()
