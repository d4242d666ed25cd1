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


def storm_batch(scen, warm):
    """A plain FP32 Batch of (params, zb, boundary) scenarios, set up from
    their boundaries and beds and advanced `warm` coupled steps."""
    from .model import Batch
    b = Batch([p for p, _, _ in scen])
    for s, (p, zb, bnd) in enumerate(scen):
        m = b.scenario(s)
        m.set_wave_boundary(0, bnd["St"], bnd["q"], t0=0.0, tend=p.rtlength, Trep=bnd["Trep"])
        m.set_sealevel([0.0, 1e6], [0.0, 0.0], [0.0, 0.0])
        m.set_wind([0.0, 1e6], [0.0, 0.0], [0.0, 0.0])
        m.init_state(zb, 0.0, 0.0)
    b.advance(warm)
    b.sync()
    return b


def collect_batch(scen, warm=200, every=20, count=6, k=10, crop=160, crops_per=4, seed=0):
    """Snapshot pairs from a plain batched run of (params, zb, boundary)
    scenarios (the storm ensemble: boundary["storm"] gives Hm0, Tp at model
    time t): at each snapshot, crops_per windows of crop x crop cells per
    scenario around its shoreline (x from 55 % to 85 % of the cross-shore
    extent) of the inputs and held wave fields at t, and of the wave fields
    at t + k in the same windows.  Returns dict(x, y, hold) as collect()."""
    b = storm_batch(scen, warm)
    rng = np.random.default_rng(seed)
    xs, ys, hs = [], [], []
    for _ in range(count):
        t = b.status()["t"]
        wins = []
        for s, (p, zb, bnd) in enumerate(scen):
            m = b.scenario(s)
            hs_, tp_ = bnd["storm"](float(t[s]))
            fin = np.stack([m.get(f).reshape(p.ny, p.nx) for f in IN_FIELDS] +
                           [np.full((p.ny, p.nx), hs_, np.float32), np.full((p.ny, p.nx), tp_, np.float32)], -1)
            hold = np.stack([m.get(f).reshape(p.ny, p.nx) for f in OUT_FIELDS], -1)
            z = np.zeros((p.ny, p.nx, IN_CH - len(IN_FIELDS) - 2 - OUT_CH), np.float32)
            x = np.concatenate([fin, hold, z], -1).astype(np.float32)
            for _c in range(crops_per):
                lo = max(0, int(0.55 * p.nx) - crop // 2)
                hi = max(lo, min(p.nx - crop, int(0.85 * p.nx) - crop // 2))
                x0 = int(rng.integers(lo, hi + 1))
                y0 = int(rng.integers(0, p.ny - crop + 1))
                wins.append((s, y0, x0))
                xs.append(x[y0:y0 + crop, x0:x0 + crop])
                hs.append(hold[y0:y0 + crop, x0:x0 + crop].astype(np.float32))
        b.advance(k)
        cache = {}
        for s, y0, x0 in wins:
            p = scen[s][0]
            if s not in cache:
                m = b.scenario(s)
                cache[s] = np.stack([m.get(f).reshape(p.ny, p.nx) for f in OUT_FIELDS], -1)
            ys.append(cache[s][y0:y0 + crop, x0:x0 + crop].astype(np.float32))
        b.advance(max(0, every - k))
    b.close()
    return dict(x=np.stack(xs), y=np.stack(ys), hold=np.stack(hs))


class CropRecorder:
    """Training pairs from the states a surrogate-assisted batch actually
    visits (push-forward data): around each judge segment of a
    BatchSurrogateRun, crops_per windows per scenario of the inputs and held
    fields before the segment's k plain steps and of the wave fields after
    them (windows around the shoreline as in collect_batch)."""

    def __init__(self, batch, scen, crop=96, crops_per=2, seed=0):
        self.b, self.scen, self.crop, self.crops_per = batch, scen, crop, crops_per
        self.rng = np.random.default_rng(seed)
        self.xs, self.ys, self.hs = [], [], []
        self.wins = []

    def before(self, t):
        crop = self.crop
        self.wins = []
        for s, (p, zb, bnd) in enumerate(self.scen):
            m = self.b.scenario(s)
            hs_, tp_ = bnd["storm"](t)
            fin = np.stack([m.get(f).reshape(p.ny, p.nx) for f in IN_FIELDS] +
                           [np.full((p.ny, p.nx), hs_, np.float32), np.full((p.ny, p.nx), tp_, np.float32)], -1)
            hold = np.stack([m.get(f).reshape(p.ny, p.nx) for f in OUT_FIELDS], -1)
            z = np.zeros((p.ny, p.nx, IN_CH - len(IN_FIELDS) - 2 - OUT_CH), np.float32)
            x = np.concatenate([fin, hold, z], -1).astype(np.float32)
            for _c in range(self.crops_per):
                lo = max(0, int(0.55 * p.nx) - crop // 2)
                hi = max(lo, min(p.nx - crop, int(0.85 * p.nx) - crop // 2))
                x0 = int(self.rng.integers(lo, hi + 1))
                y0 = int(self.rng.integers(0, p.ny - crop + 1))
                self.wins.append((s, y0, x0))
                self.xs.append(x[y0:y0 + crop, x0:x0 + crop])
                self.hs.append(hold[y0:y0 + crop, x0:x0 + crop].astype(np.float32))

    def after(self):
        crop, cache = self.crop, {}
        for s, y0, x0 in self.wins:
            p = self.scen[s][0]
            if s not in cache:
                m = self.b.scenario(s)
                cache[s] = np.stack([m.get(f).reshape(p.ny, p.nx) for f in OUT_FIELDS], -1)
            self.ys.append(cache[s][y0:y0 + crop, x0:x0 + crop].astype(np.float32))

    def data(self):
        return dict(x=np.stack(self.xs), y=np.stack(self.ys), hold=np.stack(self.hs))


def pushforward_data(net, norm, scen, warm=150, steps=200, k=10, judge_every=20, crop=96, crops_per=4, seed=0):
    """Training pairs against chained drift (push-forward data): the
    scenarios step surrogate-assisted with `net` and no error bar, and at
    every judge segment a CropRecorder keeps the inputs there -- whose held
    wave fields, and wave energy, are the network's own earlier predictions
    after judge_every - k forced steps -- with the plain solver's fields k
    steps on as the targets.  Training on these as well teaches the network
    to correct the drift its chained predictions leave in its inputs."""
    from .surrogate_couple import BatchSurrogateRun
    b = storm_batch(scen, warm)
    rec = CropRecorder(b, scen, crop=crop, crops_per=crops_per, seed=seed)
    run = BatchSurrogateRun(b, [p for p, _, _ in scen], net, norm, lambda s, t: scen[s][2]["storm"](t), k=k,
                            judge_every=judge_every, threshold=float("inf"), recorder=rec)
    run.advance(steps)
    b.close()
    d = rec.data()
    d["judged"] = run.judged
    return d


def collect_chain(scen, warm=150, k=10, links=8, crop=96, crops_per=4, seed=0):
    """Consecutive snapshots k steps apart of a plain batched run, in fixed
    windows (crops_per per scenario, around the shoreline as in
    collect_batch): x [links + 1, W, crop, crop, IN_CH] with the held wave
    fields at each snapshot in its last channels.  Snapshot j + 1's held
    fields are snapshot j's target, so a chain gives the plain pairs and,
    with the network's own predictions in place of the held fields, the
    push-forward pairs (pushforward_pairs)."""
    b = storm_batch(scen, warm)
    rng = np.random.default_rng(seed)
    wins = []
    for s, (p, _, _) in enumerate(scen):
        for _c in range(crops_per):
            lo = max(0, int(0.55 * p.nx) - crop // 2)
            hi = max(lo, min(p.nx - crop, int(0.85 * p.nx) - crop // 2))
            wins.append((s, int(rng.integers(0, p.ny - crop + 1)), int(rng.integers(lo, hi + 1))))
    xs = []
    for j in range(links + 1):
        t = b.status()["t"]
        cache = {}
        snap = []
        for s, y0, x0 in wins:
            if s not in cache:
                p, zb, bnd = scen[s]
                m = b.scenario(s)
                hs_, tp_ = bnd["storm"](float(t[s]))
                fin = np.stack([m.get(f).reshape(p.ny, p.nx) for f in IN_FIELDS] +
                               [np.full((p.ny, p.nx), hs_, np.float32), np.full((p.ny, p.nx), tp_, np.float32)], -1)
                hold = np.stack([m.get(f).reshape(p.ny, p.nx) for f in OUT_FIELDS], -1)
                z = np.zeros((p.ny, p.nx, IN_CH - len(IN_FIELDS) - 2 - OUT_CH), np.float32)
                cache[s] = np.concatenate([fin, hold, z], -1).astype(np.float32)
            snap.append(cache[s][y0:y0 + crop, x0:x0 + crop])
        xs.append(np.stack(snap))
        if j < links:
            b.advance(k)
    b.close()
    return np.stack(xs)


def pushforward_pairs(net, norm, chain):
    """Training pairs whose held wave fields are the network's own
    prediction (the push-forward trick against chained drift): for each link
    j of a chain, the prediction from snapshot j replaces the held fields
    (and the wave-energy input) of snapshot j + 1, whose target stays the
    plain fields at snapshot j + 2."""
    h0 = len(IN_FIELDS) + 2
    ie = IN_FIELDS.index("E")
    xs, ys, hs = [], [], []
    for j in range(chain.shape[0] - 2):
        x = chain[j]
        pred = predict(net, norm, x, x[..., h0:h0 + OUT_CH])
        xn = chain[j + 1].copy()
        xn[..., h0:h0 + OUT_CH] = pred
        xn[..., ie] = pred[..., OUT_FIELDS.index("E")]
        xs.append(xn)
        ys.append(chain[j + 2][..., h0:h0 + OUT_CH])
        hs.append(pred.astype(np.float32))
    return dict(x=np.concatenate(xs).astype(np.float32), y=np.concatenate(ys).astype(np.float32),
                hold=np.concatenate(hs))


def chain_pairs(chain):
    """The plain pairs of a chain: snapshot j's inputs, snapshot j + 1's
    held fields as the target."""
    h0 = len(IN_FIELDS) + 2
    return dict(x=np.concatenate(chain[:-1]), y=np.concatenate([c[..., h0:h0 + OUT_CH] for c in chain[1:]]),
                hold=np.concatenate([c[..., h0:h0 + OUT_CH] for c in chain[:-1]]))


def merge(*ds):
    """One training set from several of the same crop size."""
    return {k: np.concatenate([d[k] for d in ds]) for k in ("x", "y", "hold")}


class Normalizer:
    """Per-channel mean and standard deviation of the inputs and of the
    k-step changes of the wave fields (the targets)."""

    def __init__(self, data):
        self.xm = data["x"].reshape(-1, IN_CH).mean(0)
        self.xs = data["x"].reshape(-1, IN_CH).std(0) + 1e-6
        d = (data["y"] - data["hold"]).reshape(-1, OUT_CH)
        self.ym = d.mean(0)
        self.ys = d.std(0) + 1e-6

    @classmethod
    def from_stats(cls, xm, xs, ym, ys):
        n = cls.__new__(cls)
        n.xm, n.xs, n.ym, n.ys = xm, xs, ym, ys
        return n

    def x(self, a):
        return (a - self.xm) / self.xs

    def y(self, a):
        return (a - self.ym) / self.ys

    def y_inv(self, a):
        return a * self.ys + self.ym


def device_data(data, norm):
    """The normalised training set resident on the GPU: inputs bf16 [S, ny,
    nx, IN_CH] and targets (the normalised k-step changes) f32 [S, ny, nx,
    OUT_CH], built once per (data, norm)."""
    import torch
    c = data.get("_device")
    if c is None or c[0] is not norm:
        x = torch.from_numpy(np.ascontiguousarray(norm.x(data["x"]), dtype=np.float32)).cuda().bfloat16()
        y = torch.from_numpy(np.ascontiguousarray(norm.y(data["y"] - data["hold"]), dtype=np.float32)).cuda()
        c = data["_device"] = (norm, x, y)
    return c[1], c[2]


def batches(data, norm, batch, crop, rng):
    """An endless stream of (x [B*crop*crop, IN_CH] bf16, y [B*crop*crop, 6]
    f32) CUDA tensors of random crops, cut on the GPU from the resident
    normalised training set (xbg_nn_gather_crops); the crop positions come
    from rng."""
    import torch
    from .surrogate import _bind_ops, _ok, _p, lib
    L = lib()
    _bind_ops(L)
    S, ny, nx, _ = data["x"].shape
    X, Y = device_data(data, norm)
    while True:
        s = rng.integers(0, S, batch)
        y0 = rng.integers(0, ny - crop + 1, batch)
        x0 = rng.integers(0, nx - crop + 1, batch)
        idx = torch.from_numpy(np.stack([s, y0, x0], 1).astype(np.int32).ravel()).cuda()
        xt = torch.empty(batch * crop * crop, IN_CH, dtype=torch.bfloat16, device="cuda")
        yt = torch.empty(batch * crop * crop, OUT_CH, dtype=torch.float32, device="cuda")
        _ok(L.xbg_nn_gather_crops(_p(X), _p(xt), _p(idx), batch, ny, nx, crop, IN_CH * 2, None), "crops x")
        _ok(L.xbg_nn_gather_crops(_p(Y), _p(yt), _p(idx), batch, ny, nx, crop, OUT_CH * 4, None), "crops y")
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


class DeviceSet:
    """The surrogate's training set kept on the GPU at its stated size:
    snapshot pairs of config-2-style runs (barred beaches at full domain
    size), copied from the model planes on the device after each snapshot
    (xbg_nn_copy_planes; nothing crosses to the host), then normalised into
    one bf16 channel-last input tensor [S, ny, nx, IN_CH] (xbg_nn_encode)
    and one f32 target tensor [S, ny, nx, 6] of the normalised k-step
    changes.  The dataset is `pairs` crops of crop x crop cells drawn once
    from the snapshot pairs (seeded); epochs walk it in shuffled batches,
    cut on the device (xbg_nn_gather_crops)."""

    def __init__(self, nx=1024, ny=512, seeds=tuple(range(8)), Hs_list=(1.5, 2.5, 3.5), warm=300, every=20,
                 count=20, k=10, pairs=20000, crop=256, seed=0):
        import torch
        from .abi import XBG_FP32
        from .model import Model
        from .scenarios import make_case, wave_group_boundary
        from .surrogate import _bind_ops, _ok, _p, lib
        L = lib()
        _bind_ops(L)
        P = nx * ny
        runs = [(sd, hs) for sd in seeds for hs in Hs_list]
        S = len(runs) * count
        raw = torch.empty(S, IN_CH + OUT_CH, P, dtype=torch.float32, device="cuda")   # inputs, then y at t + k
        raw[:, len(IN_FIELDS):len(IN_FIELDS) + 2].zero_()
        raw[:, IN_CH - (IN_CH - len(IN_FIELDS) - 2 - OUT_CH):IN_CH].zero_()
        j = 0
        for sd, hs in runs:
            p, zb, bnd = make_case("barred_beach", seed=sd, nx=nx, ny=ny)
            St, q = wave_group_boundary(p, bnd["St"].shape[0], hs, bnd["Tp"], 10 * np.pi / 180, seed=sd + 1)
            m = Model(p, XBG_FP32)
            m.set_wave_boundary(0, St, q, t0=0.0, tend=p.rtlength, Trep=bnd["Trep"])
            m.set_sealevel([0.0, 1e6], [0.0, 0.0], [0.0, 0.0])
            m.set_wind([0.0, 1e6], [0.0, 0.0], [0.0, 0.0])
            m.init_state(zb, 0.0, 0.0)
            m.advance(warm)
            src_in = [m.device_ptr(f)[0] for f in IN_FIELDS]
            src_out = [m.device_ptr(f)[0] for f in OUT_FIELDS]
            for _ in range(count):
                m.sync()
                row = raw[j]
                dst = [row[c].data_ptr() for c in range(len(IN_FIELDS))] + \
                      [row[len(IN_FIELDS) + 2 + c].data_ptr() for c in range(OUT_CH)]
                src = torch.tensor(src_in + src_out, dtype=torch.int64, device="cuda")
                dstt = torch.tensor(dst, dtype=torch.int64, device="cuda")
                _ok(L.xbg_nn_copy_planes(_p(src), _p(dstt), len(dst), P, None), "copy planes")
                row[len(IN_FIELDS)].fill_(float(hs))
                row[len(IN_FIELDS) + 1].fill_(float(bnd["Tp"]))
                torch.cuda.synchronize()
                m.advance(k)
                m.sync()
                srcy = torch.tensor(src_out, dtype=torch.int64, device="cuda")
                dsty = torch.tensor([row[IN_CH + c].data_ptr() for c in range(OUT_CH)], dtype=torch.int64,
                                    device="cuda")
                _ok(L.xbg_nn_copy_planes(_p(srcy), _p(dsty), OUT_CH, P, None), "copy planes")
                torch.cuda.synchronize()
                m.advance(max(0, every - k))
                j += 1
            m.close()
        hold = raw[:, len(IN_FIELDS) + 2:len(IN_FIELDS) + 2 + OUT_CH]
        dy = raw[:, IN_CH:] - hold
        xm = raw[:, :IN_CH].mean(dim=(0, 2)).double().cpu().numpy()
        xs = raw[:, :IN_CH].std(dim=(0, 2)).double().cpu().numpy() + 1e-6
        ym = dy.mean(dim=(0, 2)).double().cpu().numpy()
        ys = dy.std(dim=(0, 2)).double().cpu().numpy() + 1e-6
        self.norm = Normalizer.from_stats(xm, xs, ym, ys)
        # inputs: normalised bf16, channel-last, by the library's encoder
        self.X = torch.empty(S, ny, nx, IN_CH, dtype=torch.bfloat16, device="cuda")
        mean = torch.from_numpy(xm.astype(np.float32)).cuda()
        istd = torch.from_numpy((1.0 / xs).astype(np.float32)).cuda()
        for t in range(S):
            planes = torch.tensor([raw[t, c].data_ptr() for c in range(IN_CH)], dtype=torch.int64, device="cuda")
            _ok(L.xbg_nn_encode(_p(planes), IN_CH, _p(mean), _p(istd), _p(self.X[t]), P, None), "encode")
        # targets: normalised changes, channel-last f32 (data loading, on the device)
        self.Y = ((dy - torch.from_numpy(ym.astype(np.float32)).cuda()[None, :, None]) /
                  torch.from_numpy(ys.astype(np.float32)).cuda()[None, :, None]).permute(0, 2, 1).contiguous()
        self.Y = self.Y.view(S, ny, nx, OUT_CH)
        self.hold_raw = raw[:, len(IN_FIELDS) + 2:len(IN_FIELDS) + 2 + OUT_CH]
        self.y_raw = raw[:, IN_CH:]
        self.raw = raw
        self.S, self.ny, self.nx, self.crop, self.k = S, ny, nx, crop, k
        rng = np.random.default_rng(seed)
        self.pairs = np.stack([rng.integers(0, S, pairs), rng.integers(0, ny - crop + 1, pairs),
                               rng.integers(0, nx - crop + 1, pairs)], 1).astype(np.int32)

    def epoch(self, batch, rng):
        """Batches (x [B*crop*crop, IN_CH] bf16, y [B*crop*crop, 6] f32) over
        the dataset's crops in a shuffled order (the last partial batch left
        out)."""
        import torch
        from .surrogate import _ok, _p, lib
        L = lib()
        order = rng.permutation(len(self.pairs))
        c = self.crop
        xt = torch.empty(batch * c * c, IN_CH, dtype=torch.bfloat16, device="cuda")
        yt = torch.empty(batch * c * c, OUT_CH, dtype=torch.float32, device="cuda")
        for b0 in range(0, len(order) - batch + 1, batch):
            idx = torch.from_numpy(self.pairs[order[b0:b0 + batch]].ravel()).cuda()
            _ok(L.xbg_nn_gather_crops(_p(self.X), _p(xt), _p(idx), batch, self.ny, self.nx, c, IN_CH * 2, None),
                "crops x")
            _ok(L.xbg_nn_gather_crops(_p(self.Y), _p(yt), _p(idx), batch, self.ny, self.nx, c, OUT_CH * 4, None),
                "crops y")
            yield xt, yt


def train_set(net, ds, epochs=3, batch=64, lr=1e-3, seed=0, log_every=100):
    """Adam over `epochs` passes of a DeviceSet; returns the loss history."""
    rng = np.random.default_rng(seed)
    hist, k = [], 0
    for _e in range(epochs):
        for xt, yt in ds.epoch(batch, rng):
            loss = net.train_step(xt, yt, batch, ds.crop, ds.crop, lr=lr)
            k += 1
            if k % log_every == 0:
                hist.append((k, float(loss.item())))
    hist.append((k, float(loss.item())))
    net.check()
    return hist


def evaluate_fp64(net, norm, nx=1024, ny=512, seed=11, Hs=2.2, warm=300, k=10, count=3, every=20):
    """Full-domain inference on a held-out beach against the plain wave
    solver of the FP64 build: from each of `count` states of the FP64 run
    (its inputs rounded to float for the network), the prediction k steps on
    and the held fields, both against the FP64 plain result; relative L2
    errors per output field, worst over the states."""
    from .abi import XBG_FP64
    from .model import Model
    from .scenarios import make_case, wave_group_boundary
    p, zb, bnd = make_case("barred_beach", seed=seed, nx=nx, ny=ny)
    St, q = wave_group_boundary(p, bnd["St"].shape[0], Hs, bnd["Tp"], 10 * np.pi / 180, seed=seed + 1)
    m = Model(p, XBG_FP64)
    m.set_wave_boundary(0, St, q, t0=0.0, tend=p.rtlength, Trep=bnd["Trep"])
    m.set_sealevel([0.0, 1e6], [0.0, 0.0], [0.0, 0.0])
    m.set_wind([0.0, 1e6], [0.0, 0.0], [0.0, 0.0])
    m.init_state(zb, 0.0, 0.0)
    m.advance(warm)
    out = {f: dict(surrogate=0.0, hold=0.0) for f in OUT_FIELDS}
    for _ in range(count):
        h = np.stack([m.get(f).reshape(ny, nx) for f in OUT_FIELDS], -1)
        z = np.zeros((ny, nx, IN_CH - len(IN_FIELDS) - 2 - OUT_CH))
        x = np.concatenate([np.stack([m.get(f).reshape(ny, nx) for f in IN_FIELDS] +
                                     [np.full((ny, nx), Hs), np.full((ny, nx), bnd["Tp"])], -1), h, z], -1)
        pred = predict(net, norm, x[None].astype(np.float32), h[None].astype(np.float32))[0].astype(np.float64)
        m.advance(k)
        y = np.stack([m.get(f).reshape(ny, nx) for f in OUT_FIELDS], -1)
        for c, f in enumerate(OUT_FIELDS):
            out[f]["surrogate"] = max(out[f]["surrogate"], rel_err(pred[..., c], y[..., c]))
            out[f]["hold"] = max(out[f]["hold"], rel_err(h[..., c], y[..., c]))
        m.advance(max(0, every - k))
    m.close()
    return out


def conv_flops(net, B, H, W):
    """Useful FLOPs of one forward pass (the 3x3 convolutions, by level)."""
    scale = {"e1": 1, "e2": 2, "e3": 4, "e4": 8, "d3": 4, "d2": 2, "d1": 1, "he": 1}
    return sum(2 * (H // scale[n[:2]]) * (W // scale[n[:2]]) * B * l.cout * 9 * l.cin for n, l in net.L.items())


def time_training(B, H, W, steps=10, warmup=3, base=32, implicit=True, seed=1):
    """CUDA-event times of UNet.forward and UNet.train_step on a seeded random
    batch of B crops of H x W: (forward ms, train ms, forward TFLOP/s, train
    TFLOP/s); a training step does three times the forward's convolution
    FLOPs (forward, input and weight gradients)."""
    import torch
    from .surrogate import UNet
    net = UNet(seed=seed, base=base)
    net.implicit_bwd = implicit
    g = torch.Generator(device="cuda").manual_seed(seed + 2)
    x = torch.randn(B * H * W, IN_CH, device="cuda", generator=g).bfloat16()
    tgt = torch.randn(B * H * W, OUT_CH, device="cuda", generator=g)
    for _ in range(warmup):
        net.train_step(x, tgt, B, H, W)
    torch.cuda.synchronize()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    ev[0].record()
    for _ in range(steps):
        net.forward(x, B, H, W)
    ev[1].record()
    for _ in range(steps):
        net.train_step(x, tgt, B, H, W)
    ev[2].record()
    torch.cuda.synchronize()
    net.check()
    fw = ev[0].elapsed_time(ev[1]) / steps
    tr = ev[1].elapsed_time(ev[2]) / steps
    fl = conv_flops(net, B, H, W)
    return fw, tr, fl / fw / 1e9, 3 * fl / tr / 1e9


def main(argv=None):
    """python -m xbeach_gpu_b200.surrogate_train time B H W [--steps S]
    [--warmup W] [--base C] [--explicit]: times the surrogate's forward pass
    and training step (the workload of the training profiles)."""
    import argparse
    ap = argparse.ArgumentParser(prog="python -m xbeach_gpu_b200.surrogate_train")
    sub = ap.add_subparsers(dest="cmd", required=True)
    t = sub.add_parser("time", help="time forward and training step on random crops")
    t.add_argument("B", type=int)
    t.add_argument("H", type=int)
    t.add_argument("W", type=int)
    t.add_argument("--steps", type=int, default=10)
    t.add_argument("--warmup", type=int, default=3)
    t.add_argument("--base", type=int, default=32)
    t.add_argument("--explicit", action="store_true", help="im2col / split-K GEMM backward")
    c = sub.add_parser("config4", help="train at the stated size (20,000 pairs of 256x256 crops, batch 64) "
                                        "and check inference against the FP64 build")
    c.add_argument("--pairs", type=int, default=20000)
    c.add_argument("--batch", type=int, default=64)
    c.add_argument("--crop", type=int, default=256)
    c.add_argument("--epochs", type=int, default=3)
    c.add_argument("--lr", type=float, default=1e-3)
    c.add_argument("--base", type=int, default=32)
    c.add_argument("--runs-seeds", type=int, default=8)
    c.add_argument("--count", type=int, default=20)
    a = ap.parse_args(argv)
    if a.cmd == "time":
        fw, tr, tf_fw, tf_tr = time_training(a.B, a.H, a.W, a.steps, a.warmup, a.base, not a.explicit)
        print(f"{'explicit' if a.explicit else 'implicit'} backward, B={a.B} H={a.H} W={a.W} base={a.base}: "
              f"forward {fw:.3f} ms ({tf_fw:.1f} TFLOP/s), training step {tr:.3f} ms ({tf_tr:.1f} TFLOP/s)")
        return
    import json
    import time
    import torch
    from .surrogate import UNet
    t0 = time.perf_counter()
    ds = DeviceSet(seeds=tuple(range(a.runs_seeds)), count=a.count, pairs=a.pairs, crop=a.crop)
    t_collect = time.perf_counter() - t0
    net = UNet(seed=0, base=a.base)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    hist = train_set(net, ds, epochs=a.epochs, batch=a.batch, lr=a.lr)
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t0
    steps = hist[-1][0]
    flops = 3 * conv_flops(net, a.batch, a.crop, a.crop) * steps
    ev = evaluate_fp64(net, ds.norm)
    print(json.dumps({"snapshot_pairs_full_domain": ds.S, "crop_pairs": len(ds.pairs), "crop": a.crop,
                      "batch": a.batch, "epochs": a.epochs, "steps": steps, "collect_s": t_collect,
                      "train_s": t_train, "train_tflops": flops / t_train / 1e12, "loss": hist,
                      "fp64_check_rel_l2": ev}))


if __name__ == "__main__":
    main()
