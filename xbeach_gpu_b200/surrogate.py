"""Python side of the wave surrogate: bindings of include/xbg_nn.h (device
kernels in libxbg_b200.so) over torch-allocated device buffers.  torch only
holds memory and streams here; every arithmetic operation of the network is
one of the library's kernels."""
import ctypes as C

from .model import load

XBG_NN_RELU = 1
XBG_NN_OUT_BF16 = 2
XBG_NN_ATOMIC = 4

_nn = None


def lib():
    """libxbg_b200.so with the xbg_nn_* signatures set."""
    global _nn
    if _nn is not None:
        return _nn
    L = load()
    vp, ip = C.c_void_p, C.c_int
    L.xbg_nn_gemm.argtypes = [vp, vp, vp, vp, ip, ip, ip, ip, ip, ip, ip, ip, vp, vp]
    _nn = L
    return L


def _p(t):
    return None if t is None else C.c_void_p(t.data_ptr())


def gemm(A, B, C_out, bias=None, relu=False, err=None, stream=None, ksplit=1):
    """C_out[M, N] = act(A[M, K] @ B[N, K]^T + bias) on the tensor cores.
    A, B: bf16 CUDA tensors (row-major, K contiguous); C_out f32 or bf16.
    ksplit > 1: C_out (f32) += A @ B^T, K split over ksplit CTAs."""
    import torch
    L = lib()
    M, K = A.shape
    N = B.shape[0]
    flags = (XBG_NN_RELU if relu else 0) | (XBG_NN_OUT_BF16 if C_out.dtype == torch.bfloat16 else 0)
    if ksplit > 1:
        flags = XBG_NN_ATOMIC
    if err is None:
        err = torch.zeros(1, dtype=torch.int32, device=A.device)
    st = None if stream is None else C.c_void_p(stream)
    rc = L.xbg_nn_gemm(_p(A), _p(B), _p(bias), _p(C_out), M, N, K, A.stride(0), B.stride(0), C_out.stride(0),
                       flags, ksplit, _p(err), st)
    if rc != 0:
        raise RuntimeError(f"xbg_nn_gemm: status {rc}")
    return err
