"""The surrogate's C ABI on a CPU-only machine: every entry point that
include/xbg_nn.h declares is exported, the new training entry points refuse
bad arguments before any CUDA call, and the host-side helpers that size
their launches agree with the kernels' rules (no GPU call is made here)."""
import ctypes as C
import os
import re

import pytest

from xbeach_gpu_b200 import model

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
XBG_ERR_ARG = 1


@pytest.fixture(scope="module")
def lib():
    from xbeach_gpu_b200 import build
    from xbeach_gpu_b200 import surrogate as sg
    build.build(verbose=False)
    L = sg.lib()
    sg._bind_ops(L)
    return L


def test_exports_every_nn_symbol(lib):
    txt = open(os.path.join(ROOT, "include", "xbg_nn.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    syms = sorted(set(re.findall(r"\b(xbg_nn_[a-z0-9_]+)\s*\(", txt)))
    assert len(syms) >= 20
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing


def test_wgrad_work_size(lib):
    # ksplit slices of N rows of 9*cin k values plus the bias row, padded to 8
    for cin, N, ks in ((16, 16, 1), (96, 32, 85), (384, 128, 22)):
        assert lib.xbg_nn_conv3x3_wgrad_work(cin, N, ks) == ks * N * (9 * cin + 8)


def test_training_entry_points_refuse_bad_arguments(lib):
    vp = C.c_void_p
    one = vp(16)   # never dereferenced: every call below fails its argument check first
    # null input, then a channel count the 16-byte copies cannot serve, then an unsupported width
    assert lib.xbg_nn_conv3x3_wgrad(None, one, one, None, one, 1, 8, 8, 16, 16, 16, 16, 144, 1, 1, one,
                                    None) == XBG_ERR_ARG
    assert lib.xbg_nn_conv3x3_wgrad(one, one, one, None, one, 1, 8, 8, 12, 16, 16, 16, 144, 1, 1, one,
                                    None) == XBG_ERR_ARG
    assert lib.xbg_nn_conv3x3_wgrad(one, one, one, None, one, 1, 8, 8, 16, 16, 24, 24, 144, 1, 1, one,
                                    None) == XBG_ERR_ARG
    assert lib.xbg_nn_conv3x3_wgrad(one, one, one, None, one, 1, 8, 8, 16, 16, 16, 16, 144, 0, 1, one,
                                    None) == XBG_ERR_ARG
    assert lib.xbg_nn_conv3x3_flip(None, 192, 16, 16, one, 192, None) == XBG_ERR_ARG
    assert lib.xbg_nn_conv3x3_flip(one, 100, 16, 16, one, 192, None) == XBG_ERR_ARG     # ldw < 9 cin
    assert lib.xbg_nn_gather_crops(None, one, one, 1, 8, 8, 4, 32, None) == XBG_ERR_ARG
    assert lib.xbg_nn_gather_crops(one, one, one, 1, 8, 8, 9, 32, None) == XBG_ERR_ARG  # crop > image
    assert lib.xbg_nn_gather_crops(one, one, one, 1, 8, 8, 4, 6, None) == XBG_ERR_ARG   # not whole words
    assert lib.xbg_nn_mse(None, None, None, None, 1, 6, 16, 64, None) == XBG_ERR_ARG


def test_forcing_steps_refuses_a_null_handle():
    L = model.load()
    L.xbg_forcing_steps.argtypes = [C.c_void_p, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p), C.c_int]
    planes = (C.c_void_p * 6)(*([C.c_void_p(16)] * 6))
    assert L.xbg_forcing_steps(None, planes, planes, 10) == XBG_ERR_ARG


def test_output_channel_slices():
    from xbeach_gpu_b200.surrogate import GEMM_N, _nslices
    for n in (16, 32, 48, 96, 192, 256, 384, 512, 640):
        sl = _nslices(n)
        assert sum(sl) == n and all(s in GEMM_N for s in sl)
        assert sl == sorted(sl, reverse=True)
    assert _nslices(384) == [256, 128]


def test_wgrad_split_bounds():
    from xbeach_gpu_b200.surrogate import wgrad_split
    # at least eight 64-pixel chunks per range, about four CTAs per SM over the k tiles
    assert wgrad_split(64 * 8, 32, 32) == 1
    assert wgrad_split(262144, 32, 32) == (4 * 148 + 2) // 3
    for P, cin in ((100, 16), (4096, 256), (262144, 96), (1 << 22, 384)):
        ks = wgrad_split(P, cin, 64)
        chunks = (P + 63) // 64
        assert 1 <= ks <= max(1, chunks // 8)
