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
