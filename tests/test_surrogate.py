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
