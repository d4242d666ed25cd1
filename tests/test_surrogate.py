"""The wave surrogate's network on the GPU (tensor-core GEMM + the kernels of
nn_ops.cu) against the same network on the CPU in float64 (torch autograd on
the CPU is the gradient oracle), with the GPU network's own bf16 weights and
input.  bf16 activations and gradients between layers bound the agreement:
forward output within 5e-2 relative L2 error, every layer's weight and bias
gradient within 8e-2 (the first layer's gradient passes through all fifteen
layers' bf16 roundings), cosine similarity above 0.995 throughout."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _cpu_reference(net, x_bf16, tgt, B, H, W):
    """Forward + backward of the same U-Net in float64 on the CPU."""
    import torch
    import torch.nn.functional as F
    from xbeach_gpu_b200.surrogate import IN_CH, OUT_CH
    c1, c2, c3, c4 = net.c
    Wt, bt = {}, {}
    for name, l in net.L.items():
        w = l.wb.float().cpu().double()[:l.cout, :9 * l.cin]                 # [cout, tap*cin + c]
        w = w.view(l.cout, 9, l.cin).permute(0, 2, 1).reshape(l.cout, l.cin, 3, 3)
        Wt[name] = w.clone().requires_grad_(True)
        bt[name] = l.b.cpu().double()[:l.cout].clone().requires_grad_(True)
    x = x_bf16.float().cpu().double().view(B, H, W, IN_CH).permute(0, 3, 1, 2)

    def conv(n, t, relu=True):
        y = F.conv2d(t, Wt[n], bt[n], padding=1)
        return F.relu(y) if relu else y

    def up(t):
        return F.interpolate(t, scale_factor=2, mode="nearest")

    e1 = conv("e1b", conv("e1a", x))
    e2 = conv("e2b", conv("e2a", F.avg_pool2d(e1, 2)))
    e3 = conv("e3b", conv("e3a", F.avg_pool2d(e2, 2)))
    e4 = conv("e4b", conv("e4a", F.avg_pool2d(e3, 2)))
    d3 = conv("d3b", conv("d3a", torch.cat([up(e4), e3], 1)))
    d2 = conv("d2b", conv("d2a", torch.cat([up(d3), e2], 1)))
    d1 = conv("d1b", conv("d1a", torch.cat([up(d2), e1], 1)))
    out = conv("head", d1, relu=False)                                       # [B, 6, H, W]
    t = tgt.cpu().double().view(B, H, W, OUT_CH).permute(0, 3, 1, 2)
    loss = ((out - t) ** 2).mean()
    loss.backward()
    gw = {}
    for name, l in net.L.items():
        g = Wt[name].grad.reshape(l.cout, l.cin, 9).permute(0, 2, 1).reshape(l.cout, 9 * l.cin)
        gw[name] = (g, bt[name].grad)
    return out.permute(0, 2, 3, 1).reshape(-1, OUT_CH).detach(), loss.item(), gw


def _rel(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)), \
        float(a @ b / max(np.linalg.norm(a) * np.linalg.norm(b), 1e-30))


def test_unet_forward_and_gradients_vs_cpu_fp64():
    import torch
    from xbeach_gpu_b200.surrogate import IN_CH, OUT_CH, UNet
    B, H, W = 2, 32, 32
    net = UNet(seed=3, base=16)
    g = torch.Generator(device="cuda").manual_seed(7)
    x = torch.randn(B * H * W, IN_CH, device="cuda", generator=g).bfloat16()
    tgt = torch.randn(B * H * W, OUT_CH, device="cuda", generator=g)
    net.zero_grad()
    out = net.forward(x, B, H, W)
    loss, dout = net.loss_grad(out, tgt, B * H * W)
    net.backward(dout, B, H, W)
    net.check()
    ref_out, ref_loss, ref_g = _cpu_reference(net, x, tgt, B, H, W)
    e, cos = _rel(out[:, :OUT_CH].cpu(), ref_out)
    assert e < 5e-2 and cos > 0.995, (e, cos)
    assert abs(loss.item() - ref_loss) <= 5e-2 * ref_loss
    bad = {}
    for name, l in net.L.items():
        gw = l.gw.cpu()[:l.cout, :9 * l.cin]
        gb = l.gb.cpu()[:l.cout]
        for what, a, b in (("w", gw, ref_g[name][0]), ("b", gb, ref_g[name][1])):
            e, cos = _rel(a, b)
            if not (e < 8e-2 and cos > 0.995):
                bad[(name, what)] = (round(e, 4), round(cos, 5))
    assert not bad, bad


def test_unet_training_lowers_the_loss():
    """Adam on a fixed batch (the network fits it): the loss falls."""
    import torch
    from xbeach_gpu_b200.surrogate import IN_CH, OUT_CH, UNet
    B, H, W = 4, 32, 32
    net = UNet(seed=5, base=16)
    g = torch.Generator(device="cuda").manual_seed(11)
    x = torch.randn(B * H * W, IN_CH, device="cuda", generator=g).bfloat16()
    xf = x.float().view(B, H, W, IN_CH)
    tgt = torch.stack([xf[..., 0] + xf[..., 1], xf[..., 2] * 0.5, xf[..., 3] - xf[..., 4], xf[..., 5],
                       xf[..., 6] * 0.2, -xf[..., 7]], -1).reshape(-1, OUT_CH).contiguous()
    losses = [net.train_step(x, tgt, B, H, W, lr=3e-3).item() for _ in range(150)]
    net.check()
    assert losses[-1] < 0.3 * losses[0], (losses[0], losses[-1])


def test_training_is_deterministic():
    """The implicit backward reduces its pixel ranges in a fixed order, so two
    networks trained from the same seed on the same batch end with the same
    weights bit for bit; and it agrees with the explicit backward (im2col,
    split-K GEMMs with atomic adds, col2im) to bf16 rounding."""
    import torch
    from xbeach_gpu_b200.surrogate import IN_CH, OUT_CH, UNet
    B, H, W = 2, 32, 48
    g = torch.Generator(device="cuda").manual_seed(21)
    x = torch.randn(B * H * W, IN_CH, device="cuda", generator=g).bfloat16()
    tgt = torch.randn(B * H * W, OUT_CH, device="cuda", generator=g)
    nets = [UNet(seed=4, base=16) for _ in range(2)]
    for net in nets:
        for _ in range(5):
            net.train_step(x, tgt, B, H, W, lr=1e-3)
        net.check()
    for name in nets[0].L:
        assert torch.equal(nets[0].L[name].w, nets[1].L[name].w), name
        assert torch.equal(nets[0].L[name].b, nets[1].L[name].b), name
    a, b = UNet(seed=6, base=16), UNet(seed=6, base=16)
    b.implicit_bwd = False
    for net in (a, b):
        net.zero_grad()
        out = net.forward(x, B, H, W)
        _, dout = net.loss_grad(out, tgt, B * H * W)
        net.backward(dout, B, H, W)
        net.check()
    for name in a.L:
        e, cos = _rel(a.L[name].gw.cpu(), b.L[name].gw.cpu())
        assert e < 2e-2 and cos > 0.9998, (name, e, cos)


def test_training_crops_match_host_crops():
    """The crops cut on the GPU from the resident normalised training set are
    bit for bit the crops normalised on the host (same positions)."""
    import numpy as np
    import torch
    from xbeach_gpu_b200 import surrogate_train as st
    from xbeach_gpu_b200.surrogate import IN_CH, OUT_CH
    rng = np.random.default_rng(4)
    S, ny, nx = 3, 40, 56
    data = dict(x=rng.standard_normal((S, ny, nx, IN_CH)).astype(np.float32) * 3 + 1,
                y=rng.standard_normal((S, ny, nx, OUT_CH)).astype(np.float32),
                hold=rng.standard_normal((S, ny, nx, OUT_CH)).astype(np.float32))
    norm = st.Normalizer(data)
    B, crop = 5, 24
    xt, yt = next(st.batches(data, norm, B, crop, np.random.default_rng(9)))
    r = np.random.default_rng(9)
    s, y0, x0 = r.integers(0, S, B), r.integers(0, ny - crop + 1, B), r.integers(0, nx - crop + 1, B)
    xb = np.stack([data["x"][s[i], y0[i]:y0[i] + crop, x0[i]:x0[i] + crop] for i in range(B)])
    yb = np.stack([data["y"][s[i], y0[i]:y0[i] + crop, x0[i]:x0[i] + crop] -
                   data["hold"][s[i], y0[i]:y0[i] + crop, x0[i]:x0[i] + crop] for i in range(B)])
    xr = torch.from_numpy(norm.x(xb).reshape(-1, IN_CH).astype(np.float32)).cuda().bfloat16()
    yr = torch.from_numpy(norm.y(yb).reshape(-1, OUT_CH).astype(np.float32)).cuda()
    assert torch.equal(xt, xr) and torch.equal(yt, yr)


def test_forcing_steps_graph_matches_the_calls():
    """xbg_forcing_steps (k forced steps replayed from one CUDA graph) leaves
    the model bit for bit where the same sequence of C-ABI calls made one by
    one leaves it -- dt pass, ubnd1D, forcing at j/k (rescaled at j = k),
    flow, sediment, means -- over two segments (the second a graph replay)."""
    import numpy as np
    import torch
    from xbeach_gpu_b200.surrogate_train import OUT_FIELDS, beach_model
    k = 5
    a, _ = beach_model(2.2, seed=3, nx=192, ny=96, warm=30)
    b, _ = beach_model(2.2, seed=3, nx=192, ny=96, warm=30)
    P = 192 * 96
    f0 = torch.empty(6, P, device="cuda")
    for c, f in enumerate(OUT_FIELDS):
        f0[c] = torch.from_numpy(a.get(f)).cuda()
    f1 = f0 * torch.tensor([1.08, 1.04, 0.9, 1.1, 0.95, 1.05], device="cuda")[:, None]
    p0 = [f0[c].data_ptr() for c in range(6)]
    p1 = [f1[c].data_ptr() for c in range(6)]
    torch.cuda.synchronize()
    for _ in range(2):
        for j in range(1, k + 1):
            a.compute_dt()
            a.flow_boundary()
            a.set_wave_forcing(p0, p1, j / k, rescale=(j == k))
            a.flow_step()
            a.sediment_step()
            a.accumulate_means()
        b.forcing_steps(p0, p1, k)
    a.sync()
    b.sync()
    assert a.time()[:3] == b.time()[:3]
    for f in ("zs", "uu", "vv", "hh", "zb", "qx", "qy", "E", "H", "DR", "Fx", "Fy", "C", "ee", "rr", "zsmean",
              "Hmean"):
        assert np.array_equal(a.get(f), b.get(f)), f


@pytest.fixture(scope="module")
def trained():
    """A small surrogate trained on plain runs (256 x 128 barred beaches, two
    bathymetry seeds, two wave heights) and held-out snapshots of a third
    seed and wave height."""
    from xbeach_gpu_b200 import surrogate_train as st
    from xbeach_gpu_b200.surrogate import UNet
    train_d = st.collect(nx=256, ny=128, seeds=(0, 1), Hs_list=(1.5, 3.0), warm=200, every=15, count=8, k=10)
    test_d = st.collect(nx=256, ny=128, seeds=(5,), Hs_list=(2.2,), warm=200, every=15, count=4, k=10)
    norm = st.Normalizer(train_d)
    net = UNet(seed=1, base=16)
    st.train(net, train_d, norm, steps=3000, batch=16, crop=64, lr=5e-4)
    return net, norm, test_d


def test_trained_surrogate_beats_hold_forcing(trained):
    """What the network gains over the method without it: trained on snapshot
    pairs of plain runs (k = 10 coupled steps apart), evaluated on a held-out
    bathymetry seed and wave height, its wave fields after k steps are closer
    to the plain solver's than the held fields of step t are."""
    from xbeach_gpu_b200 import surrogate_train as st
    net, norm, test_d = trained
    res, _ = st.evaluate(net, norm, test_d)
    worse = {f: r for f, r in res.items() if not r["surrogate"] < r["hold"]}
    assert not worse, res
    assert res["H"]["surrogate"] < 0.5 * res["H"]["hold"], res["H"]


def _beach(Hs, seed=5, nx=256, ny=128, warm=200):
    from xbeach_gpu_b200.surrogate_train import beach_model
    return beach_model(Hs, seed=seed, nx=nx, ny=ny, warm=warm)


def test_surrogate_run_segments_and_judges(trained):
    """100 coupled steps alternating a plain judge segment and a surrogate
    segment of k = 10 (judge every 20 steps): half of the wave sub-steps
    come from the network, every judge records the relative H error of the
    network's k-step prediction against the plain solver (measured 0.9%,
    2.0%, 1.9%, 2.1%, 2.1%: stable when every other segment is plain), the
    first one (from a plain state) is under 2%, and the run stays close to
    the plain one (measured H 3.5%, zs 0.01%).  Longer chains of surrogate
    segments drift (bench.py --workload surrogate reports them)."""
    from xbeach_gpu_b200.surrogate_couple import SurrogateRun
    net, norm, _ = trained
    a, Tp = _beach(2.2)
    b, _ = _beach(2.2)
    a.advance(100)
    run = SurrogateRun(b, net, norm, Hs=2.2, Tp=Tp, k=10, judge_every=20, threshold=0.06)
    run.advance(100)
    assert not run.fallback, run.judged
    assert run.surrogate_steps == 50 and len(run.judged) == 5
    assert run.judged[0][1] < 0.02, run.judged
    errs = {f: _rel(b.get(f), a.get(f))[0] for f in ("H", "zb", "zs")}
    assert errs["zb"] < 1e-3 and errs["zs"] < 1e-3 and errs["H"] < 0.10, errs


def test_judge_falls_back_to_the_plain_method(trained):
    """An untrained network misses the judge's 2% H bar at the first judge
    segment; the run falls back and the rest is the plain method, so the end
    state is bit for bit the plain run's."""
    import numpy as np
    from xbeach_gpu_b200.surrogate import UNet
    from xbeach_gpu_b200.surrogate_couple import SurrogateRun
    _, norm, _ = trained
    bad = UNet(seed=9, base=16)
    a, Tp = _beach(2.2)
    b, _ = _beach(2.2)
    a.advance(100)
    run = SurrogateRun(b, bad, norm, Hs=2.2, Tp=Tp, k=10, judge_every=50, threshold=0.02)
    run.advance(100)
    assert run.fallback and run.judged[0][1] > 0.02 and run.surrogate_steps == 0
    for f in ("H", "zs", "uu", "zb", "ee"):
        assert np.array_equal(b.get(f), a.get(f)), f


def test_device_set_matches_host_collection():
    """The device-resident training set (config 4's stated size runs through
    it) holds the same snapshot pairs as the host collection of the same
    runs, bit for bit, and its crops feed the training step."""
    import torch
    from xbeach_gpu_b200 import surrogate_train as st
    from xbeach_gpu_b200.surrogate import UNet
    kw = dict(nx=256, ny=128, seeds=(0,), Hs_list=(2.0,), warm=40, every=20, count=2, k=10)
    host = st.collect(**kw)
    ds = st.DeviceSet(pairs=24, crop=64, **kw)
    raw = ds.raw.cpu().numpy()
    S, ny, nx = ds.S, ds.ny, ds.nx
    assert S == host["x"].shape[0] == 2
    x = np.moveaxis(raw[:, :16].reshape(S, 16, ny, nx), 1, -1)
    y = np.moveaxis(raw[:, 16:].reshape(S, 6, ny, nx), 1, -1)
    assert np.array_equal(x, host["x"]) and np.array_equal(y, host["y"])
    net = UNet(seed=0, base=16)
    hist = st.train_set(net, ds, epochs=2, batch=8, lr=1e-3, log_every=1)
    assert len(hist) >= 6 and all(np.isfinite(v) for _, v in hist)
    torch.cuda.synchronize()
