"""Training data, training loop and evaluation of the wave surrogate.

Snapshots come from the plain CUDA model on barred-beach domains of the large
single-domain kind (seeded bathymetry noise and wave heights).  At a time t
the inputs are the planes zb, hh, uu, vv, E, R (wave and roller energy, the
prior wave state), two broadcast planes Hm0 and Tp of the offshore spectrum,
and the six wave fields E, H, D (breaking dissipation), DR (roller
dissipation), Fx, Fy at t -- the forcing that "hold forcing", the method
without the network, keeps for k steps.  The target is the change of those
six fields over k more coupled steps, so the prediction is the held forcing
plus the network's correction.  The mean wave direction is the same in every
run, so it has no plane.

Crops are cut and normalised on the host (data loading); all arithmetic of
the network and its training runs on the library's kernels
(xbeach_gpu_b200.surrogate)."""
import numpy as np

from .surrogate import IN_CH, OUT_CH

IN_FIELDS = ["zb", "hh", "uu", "vv", "E", "R"]        # + Hm0, Tp planes
OUT_FIELDS = ["E", "H", "D", "DR", "Fx", "Fy"]


def beach_model(Hs, seed=5, nx=256, ny=128, warm=200):
    """A plain FP32 model of a barred beach (seeded bathymetry, wave height
    Hs) after `warm` coupled steps; returns (model, Tp)."""
    from .abi import XBG_FP32
    from .model import Model
    from .scenarios import make_case, wave_group_boundary
    p, zb, bnd = make_case("barred_beach", seed=seed, nx=nx, ny=ny)
    St, q = wave_group_boundary(p, bnd["St"].shape[0], Hs, bnd["Tp"], 10 * np.pi / 180, seed=seed + 1)
    m = Model(p, XBG_FP32)
    m.set_wave_boundary(0, St, q, t0=0.0, tend=p.rtlength, Trep=bnd["Trep"])
    m.set_sealevel([0.0, 1e6], [0.0, 0.0], [0.0, 0.0])
    m.set_wind([0.0, 1e6], [0.0, 0.0], [0.0, 0.0])
    m.init_state(zb, 0.0, 0.0)
    m.advance(warm)
    return m, bnd["Tp"]


def collect(nx=512, ny=256, seeds=(0, 1), Hs_list=(1.5, 2.5), warm=300, every=20, count=10, k=10):
    """Run the plain model and return snapshots {x: [S, ny, nx, IN_CH],
    y: [S, ny, nx, 6] at t + k, hold: [S, ny, nx, 6] at t} (float32)."""
    from .abi import XBG_FP32
    from .model import Model
    from .scenarios import make_case, wave_group_boundary
    xs, ys, hs = [], [], []
    for seed in seeds:
        for Hs in Hs_list:
            p, zb, bnd = make_case("barred_beach", seed=seed, nx=nx, ny=ny)
            nrec = bnd["St"].shape[0]
            St, q = wave_group_boundary(p, nrec, Hs, bnd["Tp"], 10 * np.pi / 180, seed=seed + 1)
            m = Model(p, XBG_FP32)
            m.set_wave_boundary(0, St, q, t0=0.0, tend=p.rtlength, Trep=bnd["Trep"])
            m.set_sealevel([0.0, 1e6], [0.0, 0.0], [0.0, 0.0])
            m.set_wind([0.0, 1e6], [0.0, 0.0], [0.0, 0.0])
            m.init_state(zb, 0.0, 0.0)
            m.advance(warm)
            for _ in range(count):
                h = np.stack([m.get(f).reshape(ny, nx) for f in OUT_FIELDS], -1)
                z = np.zeros((ny, nx, IN_CH - len(IN_FIELDS) - 2 - OUT_CH), np.float32)
                x = np.concatenate([np.stack([m.get(f).reshape(ny, nx) for f in IN_FIELDS] +
                                             [np.full((ny, nx), Hs, np.float32),
                                              np.full((ny, nx), bnd["Tp"], np.float32)], -1), h, z], -1)
                m.advance(k)
                y = np.stack([m.get(f).reshape(ny, nx) for f in OUT_FIELDS], -1)
                xs.append(x.astype(np.float32)); ys.append(y.astype(np.float32)); hs.append(h.astype(np.float32))
                m.advance(max(0, every - k))
            m.close()
    return dict(x=np.stack(xs), y=np.stack(ys), hold=np.stack(hs))


class Normalizer:
    """Per-channel mean and standard deviation of the inputs and of the
    k-step changes of the wave fields (the targets)."""

    def __init__(self, data):
        self.xm = data["x"].reshape(-1, IN_CH).mean(0)
        self.xs = data["x"].reshape(-1, IN_CH).std(0) + 1e-6
        d = (data["y"] - data["hold"]).reshape(-1, OUT_CH)
        self.ym = d.mean(0)
        self.ys = d.std(0) + 1e-6

    def x(self, a):
        return (a - self.xm) / self.xs

    def y(self, a):
        return (a - self.ym) / self.ys

    def y_inv(self, a):
        return a * self.ys + self.ym


def batches(data, norm, batch, crop, rng):
    """An endless stream of (x [B*crop*crop, 8] bf16, y [B*crop*crop, 6] f32)
    CUDA tensors of random crops."""
    import torch
    S, ny, nx, _ = data["x"].shape
    while True:
        s = rng.integers(0, S, batch)
        y0 = rng.integers(0, ny - crop + 1, batch)
        x0 = rng.integers(0, nx - crop + 1, batch)
        xb = np.stack([data["x"][s[i], y0[i]:y0[i] + crop, x0[i]:x0[i] + crop] for i in range(batch)])
        yb = np.stack([data["y"][s[i], y0[i]:y0[i] + crop, x0[i]:x0[i] + crop] -
                       data["hold"][s[i], y0[i]:y0[i] + crop, x0[i]:x0[i] + crop] for i in range(batch)])
        xt = torch.from_numpy(norm.x(xb).reshape(-1, IN_CH).astype(np.float32)).cuda().bfloat16()
        yt = torch.from_numpy(norm.y(yb).reshape(-1, OUT_CH).astype(np.float32)).cuda()
        yield xt, yt


def train(net, data, norm, steps=400, batch=16, crop=128, lr=1e-3, seed=0, log_every=50):
    """Adam on random crops; returns the loss history (host floats)."""
    rng = np.random.default_rng(seed)
    it = batches(data, norm, batch, crop, rng)
    hist = []
    for k in range(steps):
        xt, yt = next(it)
        loss = net.train_step(xt, yt, batch, crop, crop, lr=lr)
        if (k + 1) % log_every == 0 or k == steps - 1:
            hist.append((k + 1, float(loss.item())))
    net.check()
    return hist


def predict(net, norm, x, hold):
    """Full-domain inference: the wave fields at t + k from x [S, ny, nx,
    IN_CH] and the fields at t, hold [S, ny, nx, 6] (physical units)."""
    import torch
    S, ny, nx, _ = x.shape
    out = []
    for s in range(S):
        xt = torch.from_numpy(norm.x(x[s]).reshape(-1, IN_CH).astype(np.float32)).cuda().bfloat16()
        o = net.forward(xt, 1, ny, nx)[:, :OUT_CH].float().cpu().numpy().reshape(ny, nx, OUT_CH)
        out.append(hold[s] + norm.y_inv(o))
    net.check()
    return np.stack(out)


def rel_err(a, b):
    """Relative L2 error of a against b."""
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def evaluate(net, norm, data):
    """Per output field: relative L2 error of the surrogate and of holding the
    wave fields at t, both against the plain solver at t + k."""
    pred = predict(net, norm, data["x"], data["hold"])
    out = {}
    for c, f in enumerate(OUT_FIELDS):
        out[f] = dict(surrogate=rel_err(pred[..., c], data["y"][..., c]),
                      hold=rel_err(data["hold"][..., c], data["y"][..., c]))
    return out, pred
