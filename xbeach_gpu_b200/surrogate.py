"""Python side of the wave surrogate: bindings of include/xbg_nn.h (device
kernels in libxbg_b200.so) over torch-allocated device buffers.  torch only
holds memory and streams here; every arithmetic operation of the network is
one of the library's kernels."""
import ctypes as C

from .model import load

XBG_NN_RELU = 1
XBG_NN_OUT_BF16 = 2
XBG_NN_ATOMIC = 4
XBG_NN_CHECK_TIMEOUT = 8   # check of the GEMM's time-out exit (include/xbg_nn.h)

_nn = None


def lib():
    """libxbg_b200.so with the xbg_nn_* signatures set."""
    global _nn
    if _nn is not None:
        return _nn
    L = load()
    vp, ip = C.c_void_p, C.c_int
    L.xbg_nn_gemm.argtypes = [vp, vp, vp, vp, ip, ip, ip, ip, ip, ip, ip, ip, vp, vp]
    L.xbg_nn_conv3x3.argtypes = [vp, vp, vp, vp, ip, ip, ip, ip, ip, ip, ip, ip, ip, ip, vp, vp]
    L.xbg_nn_conv3x3_wgrad.argtypes = [vp, vp, vp, vp, vp, ip, ip, ip, ip, ip, ip, ip, ip, ip, ip, vp, vp]
    L.xbg_nn_conv3x3_wgrad_work.argtypes = [ip, ip, ip]
    L.xbg_nn_conv3x3_wgrad_work.restype = C.c_longlong
    L.xbg_nn_conv_set_tma.argtypes = [ip]
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


def conv3x3(x, w, y, B, H, W, cin, bias=None, relu=False, err=None, stream=None):
    """y[P, N] = act(conv3x3(x) + bias) on the tensor cores without an im2col
    matrix: x [P, ldx] bf16 NHWC (first cin channels used), w [N, Kp] bf16
    with K = tap * cin + c, y f32 or bf16 [P, ldy]."""
    import torch
    L = lib()
    N, Kp = w.shape
    flags = (XBG_NN_RELU if relu else 0) | (XBG_NN_OUT_BF16 if y.dtype == torch.bfloat16 else 0)
    if err is None:
        err = torch.zeros(1, dtype=torch.int32, device=x.device)
    st = None if stream is None else C.c_void_p(stream)
    rc = L.xbg_nn_conv3x3(_p(x), _p(w), _p(bias), _p(y), B, H, W, cin, x.stride(0), N, Kp, w.stride(0),
                          y.stride(0), flags, _p(err), st)
    if rc != 0:
        raise RuntimeError(f"xbg_nn_conv3x3: status {rc}")
    return err


def conv3x3_wgrad(x, dz, gw, gb, work, B, H, W, cin, ksplit, err, stream=None, accumulate=True):
    """gw[n][tap*cin + c] (+)= sum_p dz[p][n] x[p + tap offset][c] and gb[n]
    (+)= sum_p dz[p][n] (n < gw.shape[0]) on the tensor cores, without an
    im2col matrix; `work` holds the ksplit partial sums (f32, at least
    xbg_nn_conv3x3_wgrad_work elements), added in a fixed order."""
    L = lib()
    N = gw.shape[0]
    need = L.xbg_nn_conv3x3_wgrad_work(cin, N, ksplit)
    if work.numel() < need:
        raise ValueError(f"wgrad work buffer {work.numel()} < {need}")
    st = None if stream is None else C.c_void_p(stream)
    rc = L.xbg_nn_conv3x3_wgrad(_p(x), _p(dz), _p(gw), _p(gb), _p(work), B, H, W, cin, x.stride(0), N,
                                dz.stride(0), gw.stride(0), ksplit, 1 if accumulate else 0, _p(err), st)
    if rc != 0:
        raise RuntimeError(f"xbg_nn_conv3x3_wgrad: status {rc}")


def wgrad_split(P, cin, N):
    """Pixel ranges of the weight-gradient kernel: about four CTAs per SM
    over the k tiles, at least eight 64-pixel chunks per range."""
    tiles = (9 * cin + 1 + 127) // 128
    chunks = (P + 63) // 64
    return max(1, min(max(1, chunks // 8), (4 * 148 + tiles - 1) // tiles, 65535))


# ---------------------------------------------------------------- network
import math  # noqa: E402

import numpy as np  # noqa: E402

IN_CH = 16           # zb, h, u, v, E, R, Hm0, Tp planes + the six wave fields at t + 2 zero planes
OUT_CH = 6           # change of E, H, D, DR, Fx, Fy over k steps
GEMM_N = (16, 32, 48, 64, 96, 128, 192, 256)


def _r64(n):
    return (n + 63) // 64 * 64


def _np_for(cout):
    for n in GEMM_N:
        if n >= cout:
            return n
    raise ValueError(cout)


def _bind_ops(L):
    vp, ip, ll, fl = C.c_void_p, C.c_int, C.c_longlong, C.c_float
    L.xbg_nn_im2col3x3.argtypes = [vp, vp, ip, ip, ip, ip, ip, ip, vp]
    L.xbg_nn_col2im3x3.argtypes = [vp, vp, ip, ip, ip, ip, ip, ip, vp]
    L.xbg_nn_transpose.argtypes = [vp, vp, ip, ip, ip, ip, vp]
    L.xbg_nn_conv3x3_flip.argtypes = [vp, ip, ip, ip, vp, ip, vp]
    L.xbg_nn_gather_crops.argtypes = [vp, vp, vp, ip, ip, ip, ip, ip, vp]
    L.xbg_nn_relu_bwd.argtypes = [vp, vp, vp, ll, vp]
    L.xbg_nn_bias_grad.argtypes = [vp, vp, ip, ip, ip, vp]
    L.xbg_nn_pool2.argtypes = [vp, vp, ip, ip, ip, ip, vp]
    L.xbg_nn_pool2_bwd.argtypes = [vp, vp, ip, ip, ip, ip, ip, vp]
    L.xbg_nn_up2.argtypes = [vp, vp, ip, ip, ip, ip, ip, ip, vp]
    L.xbg_nn_up2_bwd.argtypes = [vp, vp, ip, ip, ip, ip, ip, ip, vp]
    L.xbg_nn_chan_copy.argtypes = [vp, vp, ll, ip, ip, ip, ip, ip, vp]
    L.xbg_nn_mse.argtypes = [vp, vp, vp, vp, ip, ip, ip, ip, vp]
    L.xbg_nn_adam.argtypes = [vp, vp, vp, vp, vp, ll, fl, fl, fl, fl, ip, vp]
    L.xbg_nn_to_bf16.argtypes = [vp, vp, ll, vp]
    L.xbg_nn_encode.argtypes = [vp, ip, vp, vp, vp, ll, vp]
    L.xbg_nn_decode.argtypes = [vp, ip, vp, vp, vp, vp, ip, ll, vp]
    L.xbg_nn_copy_planes.argtypes = [vp, vp, ip, ll, vp]
    L.xbg_nn_encode_batch.argtypes = [vp, ip, vp, vp, vp, vp, vp, ip, ip, ip, vp]
    L.xbg_nn_decode_batch.argtypes = [vp, ip, vp, vp, vp, vp, vp, vp, ip, ip, ip, ip, vp]


def _ok(rc, what):
    if rc != 0:
        raise RuntimeError(f"{what}: status {rc}")


class Scratch:
    """Work buffers shared by every layer (sized on first use)."""

    def __init__(self, dev):
        self.dev = dev
        self.buf = {}

    def get(self, name, shape, dtype):
        import torch
        n = int(np.prod(shape))
        b = self.buf.get(name)
        if b is None or b.numel() < n or b.dtype != dtype:
            b = torch.empty(n, dtype=dtype, device=self.dev)
            self.buf[name] = b
        return b[:n].view(*shape)


class Conv3x3:
    """3x3 convolution (zero padding) + bias + optional ReLU on NHWC bf16."""

    def __init__(self, cin, cout, relu, rng, dev, gain=2.0):
        import torch
        self.cin, self.cout, self.relu = cin, cout, relu
        self.Kp = _r64(9 * cin)
        self.Np = _np_for(cout)          # GEMM N of the forward
        if relu and self.Np != cout:     # internal outputs are stored [P, cout]
            raise ValueError(f"hidden layer width {cout} must be one of {GEMM_N}")
        self.Nk = _r64(self.Np)          # reduction of the input-gradient GEMM
        w = np.zeros((self.Np, self.Kp), np.float32)
        std = math.sqrt(gain / (9 * cin))
        w[:cout, :9 * cin] = rng.standard_normal((cout, 9 * cin)) * std
        self.w = torch.from_numpy(w).to(dev)
        self.b = torch.zeros(self.Np, dtype=torch.float32, device=dev)
        self.wb = torch.empty(self.Np, self.Kp, dtype=torch.bfloat16, device=dev)
        self.wt = None                   # W^T (explicit backward only), built on first use
        self.Kd = _r64(9 * self.Np)      # K of the input-gradient convolution (dz has Np channels)
        self.wf = torch.zeros(cin, self.Kd, dtype=torch.bfloat16, device=dev)   # flipped weights
        self.gw = torch.zeros_like(self.w)
        self.gb = torch.zeros_like(self.b)
        self.mw, self.vw = torch.zeros_like(self.w), torch.zeros_like(self.w)
        self.mb, self.vb = torch.zeros_like(self.b), torch.zeros_like(self.b)
        self.bb = torch.empty(self.Np, dtype=torch.bfloat16, device=dev)   # unused bf16 bias copy for Adam
        self.sync_copies()

    def params(self):
        return [(self.w, self.wb, self.gw, self.mw, self.vw), (self.b, self.bb, self.gb, self.mb, self.vb)]

    def sync_copies(self):
        L = lib()
        _ok(L.xbg_nn_to_bf16(_p(self.w), _p(self.wb), self.w.numel(), None), "to_bf16")
        self.refresh_t()

    def refresh_t(self):
        """Derived bf16 weights after an update: the flipped weights of the
        input-gradient convolution (and W^T once the explicit backward has
        been used)."""
        L = lib()
        _ok(L.xbg_nn_conv3x3_flip(_p(self.wb), self.Kp, self.cin, self.Np, _p(self.wf), self.Kd, None), "flip W")
        if self.wt is not None:
            _ok(L.xbg_nn_transpose(_p(self.wb), _p(self.wt), self.Np, self.Kp, self.Kp, self.Nk, None),
                "transpose W")

    def forward(self, x, y, B, H, W, S, out_f32=False, implicit=True):
        """x [P, cin] bf16 -> y [P, cout] (bf16) or [P, Np] (f32 when out_f32).
        implicit: the implicit-GEMM convolution kernel; else im2col + GEMM
        (the same products in the same order)."""
        if implicit:
            conv3x3(x, self.wb, y, B, H, W, self.cin, bias=self.b, relu=self.relu, err=S.err)
            return
        L = lib()
        P = B * H * W
        col = S.get("col", (P, self.Kp), x.dtype)
        _ok(L.xbg_nn_im2col3x3(_p(x), _p(col), B, H, W, self.cin, self.Kp, P, None), "im2col")
        gemm(col, self.wb, y, bias=self.b, relu=self.relu, err=S.err)

    def backward(self, x, y, dy, dx, B, H, W, S, accumulate=False, need_dx=True, implicit=True,
                 accumulate_grad=True):
        """dy [P, cout] (bf16 gradient of the output; the head receives the
        loss gradient [P, >= Np], zero beyond its outputs) -> dx [P, cin] =
        the input gradient; gw, gb accumulate (are overwritten when
        accumulate_grad is False, implicit only).  implicit: the weight gradient
        and the input gradient as implicit GEMMs on the tensor cores (no
        im2col matrix; deterministic); else im2col, transposes, split-K GEMMs
        with atomic adds and col2im (dx += when accumulate)."""
        if not implicit:
            self._backward_explicit(x, y, dy, dx, B, H, W, S, accumulate, need_dx)
            return
        import torch
        if accumulate:
            raise ValueError("the implicit backward writes dx; accumulate needs implicit=False")
        L = lib()
        P = B * H * W
        if self.relu:
            t = S.get("dzc", (P, self.cout), torch.bfloat16)
            _ok(L.xbg_nn_relu_bwd(_p(dy), _p(y), _p(t), P * self.cout, None), "relu_bwd")
        else:
            t = dy
        ks = wgrad_split(P, self.cin, self.Np)
        work = S.get("wgrad", (L.xbg_nn_conv3x3_wgrad_work(self.cin, self.Np, ks),), torch.float32)
        conv3x3_wgrad(x, t, self.gw, self.gb, work, B, H, W, self.cin, ks, S.err, accumulate=accumulate_grad)
        if not need_dx:
            return
        # dx = conv3x3(dz) with the flipped weights, in output-channel slices the kernel supports
        n0 = 0
        for nb in _nslices(self.cin):
            conv3x3(t, self.wf[n0:n0 + nb], dx[:, n0:n0 + nb], B, H, W, self.Np, err=S.err)
            n0 += nb

    def _backward_explicit(self, x, y, dy, dx, B, H, W, S, accumulate, need_dx):
        import torch
        L = lib()
        if self.wt is None:
            self.wt = torch.zeros(self.Kp, self.Nk, dtype=torch.bfloat16, device=self.w.device)
            self.refresh_t()
        P = B * H * W
        Mpad = (P + 127) // 128 * 128
        # ReLU mask; the input-gradient GEMM reduces over Nk (a multiple of 64)
        # columns, so a narrower gradient goes into a zero-padded buffer.  The
        # head (no ReLU) receives the loss gradient already [P, Nk]-padded.
        if self.relu:
            t = S.get("dzc", (P, self.cout), torch.bfloat16)
            _ok(L.xbg_nn_relu_bwd(_p(dy), _p(y), _p(t), P * self.cout, None), "relu_bwd")
        else:
            t = dy
        if t.shape[1] == self.Nk:
            dz = t
        else:
            dz = S.get("dz", (P, self.Nk), torch.bfloat16)
            dz.zero_()
            _ok(L.xbg_nn_chan_copy(_p(t), _p(dz), P, self.cout, self.Nk, 0, 0, 0, None), "pad dz")
        _ok(L.xbg_nn_bias_grad(_p(dz), _p(self.gb), P, self.Np, self.Nk, None), "bias_grad")
        # dW += dz^T . col  (K = pixels, split over CTAs)
        col = S.get("col", (Mpad, self.Kp), torch.bfloat16)
        _ok(L.xbg_nn_im2col3x3(_p(x), _p(col), B, H, W, self.cin, self.Kp, Mpad, None), "im2col")
        colT = S.get("colT", (self.Kp, Mpad), torch.bfloat16)
        _ok(L.xbg_nn_transpose(_p(col), _p(colT), Mpad, self.Kp, self.Kp, Mpad, None), "transpose col")
        dzT = S.get("dzT", (self.Np, Mpad), torch.bfloat16)
        dzT.zero_()
        _ok(L.xbg_nn_transpose(_p(dz), _p(dzT), P, self.Np, self.Nk, Mpad, None), "transpose dz")
        nchunks = Mpad // 64
        n0 = 0
        for nb in _chunks(self.Kp):
            tiles = (self.Np + 127) // 128 * 1
            ks = max(1, min(nchunks, 1184 // max(1, tiles * len(_chunks(self.Kp)))))
            gemm(dzT, colT[n0:n0 + nb], self.gw[:, n0:n0 + nb], err=S.err, ksplit=ks)
            n0 += nb
        if not need_dx:
            return
        # dcol = dz . W, dx (+)= col2im(dcol)
        dcol = S.get("dcol", (P, self.Kp), torch.bfloat16)
        n0 = 0
        for nb in _chunks(self.Kp):
            gemm(dz, self.wt[n0:n0 + nb], dcol[:, n0:n0 + nb], err=S.err)
            n0 += nb
        _ok(L.xbg_nn_col2im3x3(_p(dcol), _p(dx), B, H, W, self.cin, self.Kp, 1 if accumulate else 0, None), "col2im")


def _nslices(n):
    """n (a multiple of 16) as output-channel slices of the supported widths."""
    out = []
    while n > 0:
        nb = max(g for g in GEMM_N if g <= n)
        out.append(nb)
        n -= nb
    return out


def _c8(n):
    return (n + 7) // 8 * 8


def _chunks(K):
    """K (a multiple of 64) as GEMM N-chunks of the supported sizes."""
    out = []
    while K > 0:
        for nb in (256, 192, 128, 64):
            if nb <= K:
                out.append(nb)
                K -= nb
                break
    return out


class UNet:
    """The wave surrogate: a 4-level convolutional U-Net from IN_CH input planes
    to OUT_CH output planes, `base` channels at full resolution doubling per
    level (32/64/128/256), two 3x3 convolutions + ReLU per level, 2x2 average
    pooling down, nearest 2x upsampling and skip concatenation up, a 3x3 head.
    bf16 weights and activations, fp32 accumulation (tensor cores), fp32
    master weights updated by Adam."""

    NAMES = ["e1a", "e1b", "e2a", "e2b", "e3a", "e3b", "e4a", "e4b", "d3a", "d3b", "d2a", "d2b", "d1a", "d1b",
             "head"]

    def __init__(self, seed=0, base=32, dev="cuda"):
        import torch
        _bind_ops(lib())
        rng = np.random.default_rng(seed)
        c1, c2, c3, c4 = base, 2 * base, 4 * base, 8 * base
        self.c = (c1, c2, c3, c4)
        spec = {"e1a": (IN_CH, c1), "e1b": (c1, c1), "e2a": (c1, c2), "e2b": (c2, c2), "e3a": (c2, c3),
                "e3b": (c3, c3), "e4a": (c3, c4), "e4b": (c4, c4), "d3a": (c4 + c3, c3), "d3b": (c3, c3),
                "d2a": (c3 + c2, c2), "d2b": (c2, c2), "d1a": (c2 + c1, c1), "d1b": (c1, c1), "head": (c1, OUT_CH)}
        self.L = {n: Conv3x3(ci, co, n != "head", rng, dev, gain=2.0 if n != "head" else 1.0)
                  for n, (ci, co) in spec.items()}
        self.dev = dev
        self.S = Scratch(dev)
        self.S.err = torch.zeros(1, dtype=torch.int32, device=dev)
        self.nstep = 0
        self.act = None
        self.implicit_bwd = True          # False: im2col / transposes / split-K GEMMs (for comparison)
        self._acc_grad = True

    # -- helpers
    def _new(self, P, C, dtype=None):
        import torch
        return torch.empty(P, C, dtype=dtype or torch.bfloat16, device=self.dev)

    def _conv(self, name, x, B, H, W, out_f32=False):
        import torch
        l = self.L[name]
        y = self._new(B * H * W, l.Np if out_f32 else l.cout, torch.float32 if out_f32 else None)
        l.forward(x, y, B, H, W, self.S)
        self.act[name] = (x, y, B, H, W)
        return y

    def _pool(self, x, B, H, W, C):
        y = self._new(B * (H // 2) * (W // 2), C)
        _ok(lib().xbg_nn_pool2(_p(x), _p(y), B, H, W, C, None), "pool2")
        return y

    def _cat(self, lo, hi, B, h, w, clo, chi):
        """[upsample(lo) | hi] on the fine grid (2h x 2w)."""
        P = B * 4 * h * w
        y = self._new(P, clo + chi)
        _ok(lib().xbg_nn_up2(_p(lo), _p(y), B, h, w, clo, clo + chi, 0, None), "up2")
        _ok(lib().xbg_nn_chan_copy(_p(hi), _p(y), P, chi, clo + chi, clo, 0, 0, None), "concat")
        return y

    # -- forward / backward
    def forward(self, x, B, H, W):
        """x [B*H*W, IN_CH] bf16 (NHWC) -> [B*H*W, 16] f32 (channels 0..5 used)."""
        c1, c2, c3, c4 = self.c
        self.act = {}
        H2, W2, H3, W3, H4, W4 = H // 2, W // 2, H // 4, W // 4, H // 8, W // 8
        a = self._conv("e1a", x, B, H, W)
        e1 = self._conv("e1b", a, B, H, W)
        a = self._conv("e2a", self._pool(e1, B, H, W, c1), B, H2, W2)
        e2 = self._conv("e2b", a, B, H2, W2)
        a = self._conv("e3a", self._pool(e2, B, H2, W2, c2), B, H3, W3)
        e3 = self._conv("e3b", a, B, H3, W3)
        a = self._conv("e4a", self._pool(e3, B, H3, W3, c3), B, H4, W4)
        e4 = self._conv("e4b", a, B, H4, W4)
        a = self._conv("d3a", self._cat(e4, e3, B, H4, W4, c4, c3), B, H3, W3)
        d3 = self._conv("d3b", a, B, H3, W3)
        a = self._conv("d2a", self._cat(d3, e2, B, H3, W3, c3, c2), B, H2, W2)
        d2 = self._conv("d2b", a, B, H2, W2)
        a = self._conv("d1a", self._cat(d2, e1, B, H2, W2, c2, c1), B, H, W)
        d1 = self._conv("d1b", a, B, H, W)
        return self._conv("head", d1, B, H, W, out_f32=True)

    def _bwd(self, name, dy, accumulate_into=None, need_dx=True):
        acc = self._acc_grad
        x, y, B, H, W = self.act[name]
        l = self.L[name]
        dx = accumulate_into if accumulate_into is not None else (self._new(B * H * W, l.cin) if need_dx else None)
        l.backward(x, y, dy, dx, B, H, W, self.S, accumulate=accumulate_into is not None, need_dx=need_dx,
                   implicit=self.implicit_bwd, accumulate_grad=acc)
        return dx

    def backward(self, dout, B, H, W, accumulate_grad=True):
        """dout [P, 64] bf16: gradient of the loss w.r.t. the head output.
        The weight and bias gradients are added to gw, gb (stored over them
        when accumulate_grad is False: implicit backward only)."""
        if not accumulate_grad and not self.implicit_bwd:
            raise ValueError("accumulate_grad=False needs the implicit backward")
        self._acc_grad = accumulate_grad
        c1, c2, c3, c4 = self.c
        L = lib()
        H2, W2, H3, W3, H4, W4 = H // 2, W // 2, H // 4, W // 4, H // 8, W // 8

        def split(gcat, B, h, w, clo, chi):   # -> (grad of the coarse input, grad of the skip)
            glo = self._new(B * h * w, clo)
            ghi = self._new(B * 4 * h * w, chi)
            _ok(L.xbg_nn_up2_bwd(_p(gcat), _p(glo), B, h, w, clo, clo + chi, 0, None), "up2_bwd")
            _ok(L.xbg_nn_chan_copy(_p(ghi), _p(gcat), B * 4 * h * w, chi, clo + chi, clo, 1, 0, None), "split")
            return glo, ghi

        def pool_bwd(gp, into, B, H, W, C):
            _ok(L.xbg_nn_pool2_bwd(_p(gp), _p(into), B, H, W, C, 1, None), "pool2_bwd")

        g = self._bwd("head", dout)
        g = self._bwd("d1a", self._bwd("d1b", g))
        gd2, ge1 = split(g, B, H2, W2, c2, c1)
        g = self._bwd("d2a", self._bwd("d2b", gd2))
        gd3, ge2 = split(g, B, H3, W3, c3, c2)
        g = self._bwd("d3a", self._bwd("d3b", gd3))
        ge4, ge3 = split(g, B, H4, W4, c4, c3)
        gp3 = self._bwd("e4a", self._bwd("e4b", ge4))
        pool_bwd(gp3, ge3, B, H3, W3, c3)
        gp2 = self._bwd("e3a", self._bwd("e3b", ge3))
        pool_bwd(gp2, ge2, B, H2, W2, c2)
        gp1 = self._bwd("e2a", self._bwd("e2b", ge2))
        pool_bwd(gp1, ge1, B, H, W, c1)
        self._bwd("e1a", self._bwd("e1b", ge1), need_dx=False)

    def zero_grad(self):
        for l in self.L.values():
            l.gw.zero_()
            l.gb.zero_()

    def loss_grad(self, out, tgt, P):
        """MSE of out[:, :6] against tgt [P, 6] (f32); returns (loss device
        scalar, gradient [P, 64] bf16)."""
        import torch
        loss = torch.zeros(1, dtype=torch.float32, device=self.dev)
        dout = self._new(P, 64)
        _ok(lib().xbg_nn_mse(_p(out), _p(tgt), _p(dout), _p(loss), P, OUT_CH, out.shape[1], 64, None), "mse")
        return loss, dout

    def adam(self, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
        self.nstep += 1
        L = lib()
        for l in self.L.values():
            for (p_, pb, g, m, v) in l.params():
                _ok(L.xbg_nn_adam(_p(p_), _p(pb), _p(g), _p(m), _p(v), p_.numel(), lr, b1, b2, eps, self.nstep,
                                  None), "adam")
            l.refresh_t()

    def train_step(self, x, tgt, B, H, W, lr=1e-3):
        """One Adam step on a batch; returns the loss (device scalar).  The
        implicit backward stores the gradients, so nothing is zeroed first."""
        if not self.implicit_bwd:
            self.zero_grad()
        out = self.forward(x, B, H, W)
        loss, dout = self.loss_grad(out, tgt, B * H * W)
        self.backward(dout, B, H, W, accumulate_grad=not self.implicit_bwd)
        self.adam(lr)
        return loss

    def check(self):
        """Raise if a tensor-core wait timed out in any launch so far."""
        import torch
        torch.cuda.synchronize()
        if int(self.S.err.item()) != 0:
            raise RuntimeError("tensor-core GEMM wait timed out")
