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
