"""The surrogate's tensor-core GEMM (tcgen05, bf16 in, fp32 accumulate in
tensor memory) against a plain torch fp32 matmul of the same bf16 values."""
import pytest

pytestmark = pytest.mark.gpu

SHAPES = [(128, 16, 64), (256, 32, 128), (384, 64, 192), (1000, 128, 256), (128, 256, 576), (640, 48, 64),
          (256, 96, 320), (512, 192, 128)]


@pytest.mark.parametrize("M,N,K", SHAPES)
@pytest.mark.parametrize("relu,bf16_out", [(False, False), (True, True)])
def test_gemm_vs_torch_fp32(M, N, K, relu, bf16_out):
    import torch
    from xbeach_gpu_b200 import surrogate as sg
    g = torch.Generator(device="cuda").manual_seed(M * 7 + N * 3 + K)
    A = torch.randn(M, K, device="cuda", generator=g).bfloat16()
    B = torch.randn(N, K, device="cuda", generator=g).bfloat16()
    bias = torch.randn(N, device="cuda", generator=g)
    out = torch.empty(M, N, device="cuda", dtype=torch.bfloat16 if bf16_out else torch.float32)
    err = sg.gemm(A, B, out, bias=bias, relu=relu)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    ref = A.float() @ B.float().T + bias
    if relu:
        ref = torch.relu(ref)
    tol = 2e-2 if bf16_out else 1e-3   # bf16 output rounding; fp32 accumulation order
    assert torch.allclose(out.float(), ref, rtol=tol, atol=tol * ref.abs().max().item()), \
        (out.float() - ref).abs().max().item()


@pytest.mark.parametrize("M,N,K,ks", [(128, 32, 1024, 4), (256, 64, 4096, 16), (128, 256, 640, 3)])
def test_gemm_split_k_accumulates(M, N, K, ks):
    import torch
    from xbeach_gpu_b200 import surrogate as sg
    g = torch.Generator(device="cuda").manual_seed(M + N + K)
    A = torch.randn(M, K, device="cuda", generator=g).bfloat16()
    B = torch.randn(N, K, device="cuda", generator=g).bfloat16()
    out = torch.ones(M, N, device="cuda")
    err = sg.gemm(A, B, out, ksplit=ks)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    ref = A.float() @ B.float().T + 1.0
    assert torch.allclose(out, ref, rtol=1e-3, atol=1e-3 * ref.abs().max().item())


CONV = [(1, 8, 24, 16, 32), (2, 13, 29, 32, 64), (1, 16, 16, 96, 32), (2, 9, 11, 384, 128), (1, 32, 40, 64, 256),
        (3, 7, 5, 8, 16), (1, 20, 70, 48, 192)]


@pytest.mark.parametrize("B,H,W,cin,N", CONV)
@pytest.mark.parametrize("relu,bf16_out", [(False, False), (True, True)])
def test_conv3x3_implicit_gemm(B, H, W, cin, N, relu, bf16_out):
    """The implicit-GEMM 3x3 convolution equals im2col + GEMM bit for bit (the
    same bf16 products accumulated in the same order on the tensor cores) and
    a torch fp32 convolution of the same bf16 values to fp32 accumulation
    order (bf16 output rounding when bf16)."""
    import torch
    import torch.nn.functional as F
    from xbeach_gpu_b200 import surrogate as sg
    L = sg.lib()
    sg._bind_ops(L)
    g = torch.Generator(device="cuda").manual_seed(B * 1000 + H * 31 + W * 7 + cin + N)
    P = B * H * W
    Kp = (9 * cin + 63) // 64 * 64
    x = torch.randn(P, cin, device="cuda", generator=g).bfloat16()
    w = torch.zeros(N, Kp, device="cuda", dtype=torch.bfloat16)
    w[:, :9 * cin] = (torch.randn(N, 9 * cin, device="cuda", generator=g) / (3 * cin ** 0.5)).bfloat16()
    bias = torch.randn(N, device="cuda", generator=g)
    dt = torch.bfloat16 if bf16_out else torch.float32
    y = torch.empty(P, N, device="cuda", dtype=dt)
    err = sg.conv3x3(x, w, y, B, H, W, cin, bias=bias, relu=relu)
    col = torch.empty(P, Kp, device="cuda", dtype=torch.bfloat16)
    assert L.xbg_nn_im2col3x3(sg._p(x), sg._p(col), B, H, W, cin, Kp, P, None) == 0
    y2 = torch.empty(P, N, device="cuda", dtype=dt)
    sg.gemm(col, w, y2, bias=bias, relu=relu, err=err)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    assert torch.equal(y, y2)
    wt = w[:, :9 * cin].float().view(N, 9, cin).permute(0, 2, 1).reshape(N, cin, 3, 3)
    ref = F.conv2d(x.float().view(B, H, W, cin).permute(0, 3, 1, 2), wt, bias, padding=1)
    ref = ref.permute(0, 2, 3, 1).reshape(P, N)
    if relu:
        ref = torch.relu(ref)
    tol = 2e-2 if bf16_out else 1e-3
    assert torch.allclose(y.float(), ref, rtol=tol, atol=tol * ref.abs().max().item()), \
        (y.float() - ref).abs().max().item()


def test_conv3x3_refuses_bad_layouts():
    import torch
    from xbeach_gpu_b200 import surrogate as sg
    x = torch.zeros(64, 12, device="cuda", dtype=torch.bfloat16)      # cin not a multiple of 8
    w = torch.zeros(16, 128, device="cuda", dtype=torch.bfloat16)
    y = torch.zeros(64, 16, device="cuda")
    with pytest.raises(RuntimeError):
        sg.conv3x3(x, w, y, 1, 8, 8, 12)


WGRAD = [(2, 9, 13, 16, 16, 1), (1, 16, 24, 32, 32, 3), (2, 8, 8, 48, 48, 2), (1, 12, 20, 64, 96, 5),
         (1, 8, 16, 128, 256, 2), (1, 6, 10, 384, 128, 1), (3, 7, 5, 8, 64, 4), (1, 20, 70, 96, 192, 7)]


def _wgrad_ref(x, dz, B, H, W, cin):
    """torch fp32 weight and bias gradient of the 3x3 convolution, in the
    [n][tap*cin + c] layout."""
    import torch.nn.functional as F
    P = dz.shape[0]
    xi = x.float().view(B, H, W, cin).permute(0, 3, 1, 2)
    col = F.unfold(xi, 3, padding=1)                        # [B, cin*9, H*W], index c*9 + tap
    col = col.view(B, cin, 9, H * W).permute(0, 3, 2, 1).reshape(P, 9 * cin)   # [p][tap*cin + c]
    return dz.float().t() @ col, dz.float().sum(0)


@pytest.mark.parametrize("B,H,W,cin,N,ks", WGRAD)
def test_conv3x3_wgrad_vs_torch(B, H, W, cin, N, ks):
    """The implicit weight-gradient kernel (MN-major operands, pixels as the
    reduction, a ones row for the bias) against a torch fp32 im2col matmul of
    the same bf16 values, to fp32 accumulation order; it adds into gw and gb,
    leaves the columns past 9*cin alone, and gives the same bits on a rerun
    and nearly the same with another split; without accumulate it stores."""
    import torch
    from xbeach_gpu_b200 import surrogate as sg
    L = sg.lib()
    sg._bind_ops(L)
    g = torch.Generator(device="cuda").manual_seed(B * 1000 + H * 31 + W * 7 + cin + N + ks)
    P = B * H * W
    Kp = (9 * cin + 63) // 64 * 64
    x = torch.randn(P, cin, device="cuda", generator=g).bfloat16()
    dz = torch.randn(P, N, device="cuda", generator=g).bfloat16()
    gw0 = torch.randn(N, Kp, device="cuda", generator=g)
    gb0 = torch.randn(N, device="cuda", generator=g)
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    runs = []
    for split in (ks, ks, ks + 2):
        gw, gb = gw0.clone(), gb0.clone()
        work = torch.empty(L.xbg_nn_conv3x3_wgrad_work(cin, N, split), device="cuda")
        sg.conv3x3_wgrad(x, dz, gw, gb, work, B, H, W, cin, split, err)
        runs.append((gw, gb))
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    rw, rb = _wgrad_ref(x, dz, B, H, W, cin)
    gw, gb = runs[0]
    assert torch.equal(gw[:, 9 * cin:], gw0[:, 9 * cin:])
    dw = gw[:, :9 * cin] - gw0[:, :9 * cin]
    assert torch.allclose(dw, rw, rtol=1e-4, atol=1e-4 * rw.abs().max().item()), (dw - rw).abs().max().item()
    assert torch.allclose(gb - gb0, rb, rtol=1e-4, atol=1e-4 * rb.abs().max().item())
    assert torch.equal(runs[1][0], gw) and torch.equal(runs[1][1], gb)
    assert torch.allclose(runs[2][0], gw, rtol=1e-5, atol=1e-5 * rw.abs().max().item())
    # store mode: the sums replace gw and gb (columns past 9*cin untouched)
    gs, bs = gw0.clone(), gb0.clone()
    work = torch.empty(L.xbg_nn_conv3x3_wgrad_work(cin, N, ks), device="cuda")
    sg.conv3x3_wgrad(x, dz, gs, bs, work, B, H, W, cin, ks, err, accumulate=False)
    torch.cuda.synchronize()
    assert torch.equal(gs[:, 9 * cin:], gw0[:, 9 * cin:])
    assert torch.allclose(gs[:, :9 * cin], rw, rtol=1e-4, atol=1e-4 * rw.abs().max().item())
    assert torch.allclose(bs, rb, rtol=1e-4, atol=1e-4 * rb.abs().max().item())


@pytest.mark.parametrize("B,H,W,cin,N", [(2, 9, 13, 32, 16), (1, 12, 20, 96, 64), (1, 8, 16, 384, 128),
                                         (2, 7, 5, 48, 256)])
def test_conv3x3_input_gradient_by_flipped_weights(B, H, W, cin, N):
    """The input gradient of the convolution is the convolution of dz with
    the flipped, transposed weights: xbg_nn_conv3x3_flip + xbg_nn_conv3x3
    against torch autograd of an fp32 conv2d (bf16 output rounding)."""
    import torch
    import torch.nn.functional as F
    from xbeach_gpu_b200 import surrogate as sg
    L = sg.lib()
    sg._bind_ops(L)
    g = torch.Generator(device="cuda").manual_seed(B + H + W + cin + N)
    P = B * H * W
    Kp = (9 * cin + 63) // 64 * 64
    Kd = (9 * N + 63) // 64 * 64
    w = torch.zeros(N, Kp, device="cuda", dtype=torch.bfloat16)
    w[:, :9 * cin] = (torch.randn(N, 9 * cin, device="cuda", generator=g) / (3 * cin ** 0.5)).bfloat16()
    dz = torch.randn(P, N, device="cuda", generator=g).bfloat16()
    wf = torch.full((cin, Kd), float("nan"), device="cuda", dtype=torch.bfloat16)
    assert L.xbg_nn_conv3x3_flip(sg._p(w), Kp, cin, N, sg._p(wf), Kd, None) == 0
    dx = torch.empty(P, cin, device="cuda", dtype=torch.bfloat16)
    n0 = 0
    for nb in sg._nslices(cin):
        sg.conv3x3(dz, wf[n0:n0 + nb], dx[:, n0:n0 + nb], B, H, W, N)
        n0 += nb
    torch.cuda.synchronize()
    assert not torch.isnan(wf).any()
    wt = w[:, :9 * cin].float().view(N, 9, cin).permute(0, 2, 1).reshape(N, cin, 3, 3)
    xi = torch.zeros(B, cin, H, W, device="cuda", requires_grad=True)
    F.conv2d(xi, wt, padding=1).backward(dz.float().view(B, H, W, N).permute(0, 3, 1, 2))
    ref = xi.grad.permute(0, 2, 3, 1).reshape(P, cin)
    assert torch.allclose(dx.float(), ref, rtol=2e-2, atol=2e-2 * ref.abs().max().item()), \
        (dx.float() - ref).abs().max().item()


def test_wgrad_refuses_bad_layouts():
    import torch
    from xbeach_gpu_b200 import surrogate as sg
    x = torch.zeros(64, 12, device="cuda", dtype=torch.bfloat16)      # cin not a multiple of 8
    dz = torch.zeros(64, 16, device="cuda", dtype=torch.bfloat16)
    gw = torch.zeros(16, 128, device="cuda")
    work = torch.zeros(1 << 16, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    with pytest.raises(RuntimeError):
        sg.conv3x3_wgrad(x, dz, gw, None, work, 1, 8, 8, 12, 1, err)
    x = torch.zeros(64, 16, device="cuda", dtype=torch.bfloat16)
    dz = torch.zeros(64, 24, device="cuda", dtype=torch.bfloat16)    # N = 24 unsupported
    gw = torch.zeros(24, 192, device="cuda")
    with pytest.raises(RuntimeError):
        sg.conv3x3_wgrad(x, dz, gw, None, work, 1, 8, 8, 16, 1, err)


TMA_CONV = [(2, 32, 128, 32, 32), (1, 64, 256, 16, 32), (4, 16, 64, 64, 64), (1, 8, 32, 96, 32),
            (2, 16, 16, 384, 128), (1, 16, 256, 48, 16), (2, 16, 8, 192, 64)]


@pytest.mark.parametrize("B,H,W,cin,N", TMA_CONV)
def test_conv3x3_tma_input_equals_gathered_input(B, H, W, cin, N):
    """Shapes that tile into 128-pixel row boxes take the tensor-memory-
    accelerator input path; its result equals the thread-gathered path (and
    so im2col + GEMM) bit for bit, including the zero padding at the image
    edges, between images of a batch and in the K padding."""
    import torch
    from xbeach_gpu_b200 import surrogate as sg
    L = sg.lib()
    g = torch.Generator(device="cuda").manual_seed(B * 977 + H * 31 + W * 7 + cin + N)
    P = B * H * W
    Kp = (9 * cin + 63) // 64 * 64
    ldx = cin + 8
    x = torch.randn(P, ldx, device="cuda", generator=g).bfloat16()
    w = torch.zeros(N, Kp, device="cuda", dtype=torch.bfloat16)
    w[:, :9 * cin] = (torch.randn(N, 9 * cin, device="cuda", generator=g) / (3 * cin ** 0.5)).bfloat16()
    bias = torch.randn(N, device="cuda", generator=g)
    ys = []
    for on in (1, 0):
        assert L.xbg_nn_conv_set_tma(on) == 0
        y = torch.empty(P, N, device="cuda", dtype=torch.bfloat16)
        err = sg.conv3x3(x, w, y, B, H, W, cin, bias=bias, relu=True)
        torch.cuda.synchronize()
        assert int(err.item()) == 0
        ys.append(y)
    L.xbg_nn_conv_set_tma(1)
    assert torch.equal(ys[0], ys[1])
    import torch.nn.functional as F
    wt = w[:, :9 * cin].float().view(N, 9, cin).permute(0, 2, 1).reshape(N, cin, 3, 3)
    xi = x[:, :cin].float().view(B, H, W, cin).permute(0, 3, 1, 2)
    ref = torch.relu(F.conv2d(xi, wt, bias, padding=1)).permute(0, 2, 3, 1).reshape(P, N)
    assert torch.allclose(ys[0].float(), ref, rtol=2e-2, atol=2e-2 * ref.abs().max().item())
