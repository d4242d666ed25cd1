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
