"""4-level U-Net (32/64/128/256 channels) on the library's BF16 kernels.

The network predicts a correction for the warm start of the barotropic solve
(see ``warmstart.py``).  Layers:

    enc0: conv3x3 16->32, 32->32          (input: 3 feature channels + 13 zero)
    enc1: pool, conv 32->64, 64->64
    enc2: pool, conv 64->128, 128->128
    bottom: pool, conv 128->256, 256->256
    dec2: up, conv 256->128, concat enc2, conv 256->128, 128->128
    dec1: up, conv 128->64,  concat enc1, conv 128->64, 64->64
    dec0: up, conv 64->32,   concat enc0, conv 64->32, 32->32
    head: conv1x1 32->1 (FP32)

Every convolution is followed by ReLU.  Activations and weights are BF16
(NHWC), products accumulate in FP32 on the tensor cores (the forward
convolutions and both gradients of every convolution on tcgen05 with the
accumulator in tensor memory), the master weights and Adam state are FP32.  Every arithmetic step is a kernel of
``libsevp_b200.so``; PyTorch only allocates the buffers.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import native as N

CONVS = [  # name, cin, cout
    ("enc0a", 16, 32), ("enc0b", 32, 32),
    ("enc1a", 32, 64), ("enc1b", 64, 64),
    ("enc2a", 64, 128), ("enc2b", 128, 128),
    ("bota", 128, 256), ("botb", 256, 256),
    ("up2", 256, 128), ("dec2a", 256, 128), ("dec2b", 128, 128),
    ("up1", 128, 64), ("dec1a", 128, 64), ("dec1b", 64, 64),
    ("up0", 64, 32), ("dec0a", 64, 32), ("dec0b", 32, 32),
]
HEAD_C = 32
IN_C = 16  # padded input channels (3 used)

_SIGS = {
    "sevp_nn_conv3x3": ([C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                         C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p,
                         C.c_int, C.c_int, C.c_int, C.c_void_p], C.c_int),
    "sevp_nn_conv3x3_tc": ([C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                            C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                            C.c_int, C.c_void_p], C.c_int),
    "sevp_nn_conv3x3_tma": ([C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                             C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                             C.c_int, C.c_void_p], C.c_int),
    "sevp_nn_tc_status": ([C.c_void_p], C.c_int),
    "sevp_nn_tc_set_wait_limit": ([C.c_uint], C.c_int),
    "sevp_nn_conv3x3_wgrad": ([C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int,
                               C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                               C.c_int, C.c_int, C.c_int, C.c_void_p], C.c_int),
    "sevp_nn_weight_transpose": ([C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p], C.c_int),
    "sevp_nn_weight_mirror": ([C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p], C.c_int),
    "sevp_nn_conv3x3_wgrad_tc": ([C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_int,
                                  C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p], C.c_int),
    "sevp_nn_conv3x3_backward_tc": ([C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_int,
                                     C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_void_p,
                                     C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                                     C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p], C.c_int),
    "sevp_nn_conv3x3_dgrad_tc": ([C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_int,
                                  C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int,
                                  C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p], C.c_int),
    "sevp_nn_pool": ([C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int,
                      C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p], C.c_int),
    "sevp_nn_upsample": ([C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_int,
                          C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p], C.c_int),
    "sevp_nn_head": ([C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                      C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                      C.c_longlong, C.c_int, C.c_void_p], C.c_int),
    "sevp_nn_mse": ([C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_longlong,
                     C.c_float, C.c_void_p], C.c_int),
    "sevp_nn_adam": ([C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                      C.c_longlong, C.c_float, C.c_float, C.c_float, C.c_float, C.c_int, C.c_float,
                      C.c_void_p], C.c_int),
    "sevp_nn_to_bf16": ([C.c_void_p, C.c_void_p, C.c_longlong, C.c_void_p], C.c_int),
    "sevp_nn_features": ([C.c_void_p] * 9 + [C.c_int] * 3, C.c_int),
    "sevp_nn_target": ([C.c_void_p] * 6 + [C.c_int] * 3, C.c_int),
    "sevp_nn_combine": ([C.c_void_p] * 6 + [C.c_int] * 3, C.c_int),
    "sevp_stream": ([C.c_void_p], C.c_void_p),
    "sevp_add_launches": ([C.c_void_p, C.c_int], C.c_int),
}


def lib():
    L = N.lib()
    if not getattr(L, "_nn_sigs", False):
        for name, (args, res) in _SIGS.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        L._nn_sigs = True
    return L


def _p(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


class UNet:
    """Parameters, activations and the forward/backward launch sequence for
    one input size (B, H, W); H and W must be multiples of 8."""

    def __init__(self, H: int, W: int, B: int = 1, device="cuda", seed: int = 0, stream=None,
                 train: bool = True):
        import torch

        if H % 8 or W % 8:
            raise ValueError("H and W must be multiples of 8")
        self.torch = torch
        self.dev = torch.device(device)
        self.B, self.H, self.W = B, H, W
        self.stream = stream or torch.cuda.current_stream(self.dev)
        self.sp = C.c_void_p(self.stream.cuda_stream)
        self.train = train
        self.launches = 0
        g = np.random.default_rng(seed)
        self.params = {}
        for name, cin, cout in CONVS:
            std = math.sqrt(2.0 / (9 * (3 if name == "enc0a" else cin)))
            w = g.normal(0.0, std, size=(9, cin, cout)).astype(np.float32)
            if name == "enc0a":
                w[:, 3:, :] = 0.0  # padded input channels
            self.params[name] = [torch.from_numpy(w).to(self.dev),
                                 torch.zeros(cout, dtype=torch.float32, device=self.dev)]
        hw = g.normal(0.0, 1e-3, size=(HEAD_C,)).astype(np.float32)
        self.params["head"] = [torch.from_numpy(hw).to(self.dev),
                               torch.zeros(1, dtype=torch.float32, device=self.dev)]
        self._alloc()
        self.sync_weights()
        self.step_count = 0

    # ------------------------------------------------------------ buffers
    def _alloc(self):
        torch = self.torch
        B, H, W = self.B, self.H, self.W
        P = [B * (H >> l) * (W >> l) for l in range(4)]
        self.P = P
        bf = torch.bfloat16
        z = lambda n, c: torch.zeros((n, c), dtype=bf, device=self.dev)
        A = {}
        A["x"] = z(P[0], IN_C)
        A["e0a"] = z(P[0], 32)
        A["cat0"] = z(P[0], 64)
        A["p0"] = z(P[1], 32)
        A["e1a"] = z(P[1], 64)
        A["cat1"] = z(P[1], 128)
        A["p1"] = z(P[2], 64)
        A["e2a"] = z(P[2], 128)
        A["cat2"] = z(P[2], 256)
        A["p2"] = z(P[3], 128)
        A["b0"] = z(P[3], 256)
        A["b1"] = z(P[3], 256)
        A["u2"] = z(P[2], 256)
        A["d2a"] = z(P[2], 128)
        A["d2b"] = z(P[2], 128)
        A["u1"] = z(P[1], 128)
        A["d1a"] = z(P[1], 64)
        A["d1b"] = z(P[1], 64)
        A["u0"] = z(P[0], 64)
        A["d0a"] = z(P[0], 32)
        A["d0b"] = z(P[0], 32)
        A["y"] = torch.zeros(P[0], dtype=torch.float32, device=self.dev)
        self.A = A
        self.w16 = {n: torch.zeros((9, ci, co), dtype=bf, device=self.dev) for n, ci, co in CONVS}
        # K-major ([9][co][ci]) copies: the tensor-core forward's B operand and
        # the data gradient's transposed weights
        self.wt16 = {n: torch.zeros((9, co, ci), dtype=bf, device=self.dev) for n, ci, co in CONVS}
        if self.train:
            # tap-mirrored weights ([9][ci][co]) of the tensor-core data
            # gradient, and its packed masked output gradient (the largest
            # layer has P[0] x 32 values)
            self.wm16 = {n: torch.zeros((9, ci, co), dtype=bf, device=self.dev)
                         for n, ci, co in CONVS}
            self.gscratch = torch.zeros(P[0] * 64, dtype=bf, device=self.dev)
            G = {}
            for k in ("d0b", "d0a", "d1b", "d1a", "d2b", "d2a", "b1", "b0", "e2a", "e1a", "e0a"):
                G[k] = torch.zeros_like(A[k])
            for k in ("cat0", "cat1", "cat2", "u0", "u1", "u2", "p0", "p1", "p2"):
                G[k] = torch.zeros_like(A[k])
            G["y"] = torch.zeros_like(A["y"])
            self.G = G
            self.gw = {n: [torch.zeros_like(v[0]), torch.zeros_like(v[1])] for n, v in self.params.items()}
            self.m = {n: [torch.zeros_like(v[0]), torch.zeros_like(v[1])] for n, v in self.params.items()}
            self.v = {n: [torch.zeros_like(v[0]), torch.zeros_like(v[1])] for n, v in self.params.items()}
            self.loss = torch.zeros(1, dtype=torch.float32, device=self.dev)

    def n_params(self) -> int:
        return sum(int(v[0].numel() + v[1].numel()) for v in self.params.values())

    # ------------------------------------------------------------- calls
    def _ck(self, s, what):
        if s != 0:
            raise N.SevpError(s, what)
        self.launches += 1

    def sync_weights(self):
        """BF16 working copies and their K-major transposes."""
        L = lib()
        for name, ci, co in CONVS:
            w = self.params[name][0]
            self._ck(L.sevp_nn_to_bf16(_p(w), _p(self.w16[name]), w.numel(), self.sp), "to_bf16")
            self._ck(L.sevp_nn_weight_transpose(_p(self.w16[name]), _p(self.wt16[name]), ci, co,
                                                self.sp), "transpose")
            if self.train:
                self._ck(L.sevp_nn_weight_mirror(_p(self.w16[name]), _p(self.wm16[name]), ci, co,
                                                 self.sp), "mirror")

    def _conv(self, name, src, src_off, src_ld, dst, dst_off, dst_ld, lvl):
        """Forward 3x3 conv + bias + ReLU on the tcgen05 tensor cores, operands
        loaded by TMA."""
        _, ci, co = next(c for c in CONVS if c[0] == name)
        H, W = self.H >> lvl, self.W >> lvl
        self._ck(lib().sevp_nn_conv3x3_tma(_p(src), src_ld, src_off, ci, _p(self.wt16[name]),
                                          _p(self.params[name][1]), _p(dst), dst_ld, dst_off, co,
                                          self.B, H, W, 1, self.sp), name)

    def forward(self):
        """x (features) -> y (FP32 correction).  Returns y."""
        A, L = self.A, lib()
        B, H, W = self.B, self.H, self.W
        cv = self._conv
        cv("enc0a", A["x"], 0, IN_C, A["e0a"], 0, 32, 0)
        cv("enc0b", A["e0a"], 0, 32, A["cat0"], 32, 64, 0)
        self._ck(L.sevp_nn_pool(_p(A["cat0"]), 64, 32, _p(A["p0"]), 32, 0, 32, B, H, W, 0, 0, self.sp), "pool0")
        cv("enc1a", A["p0"], 0, 32, A["e1a"], 0, 64, 1)
        cv("enc1b", A["e1a"], 0, 64, A["cat1"], 64, 128, 1)
        self._ck(L.sevp_nn_pool(_p(A["cat1"]), 128, 64, _p(A["p1"]), 64, 0, 64, B, H // 2, W // 2, 0, 0, self.sp), "pool1")
        cv("enc2a", A["p1"], 0, 64, A["e2a"], 0, 128, 2)
        cv("enc2b", A["e2a"], 0, 128, A["cat2"], 128, 256, 2)
        self._ck(L.sevp_nn_pool(_p(A["cat2"]), 256, 128, _p(A["p2"]), 128, 0, 128, B, H // 4, W // 4, 0, 0, self.sp), "pool2")
        cv("bota", A["p2"], 0, 128, A["b0"], 0, 256, 3)
        cv("botb", A["b0"], 0, 256, A["b1"], 0, 256, 3)
        self._ck(L.sevp_nn_upsample(_p(A["b1"]), 256, 0, _p(A["u2"]), 256, 0, 256, B, H // 4, W // 4, 0, self.sp), "up2")
        cv("up2", A["u2"], 0, 256, A["cat2"], 0, 256, 2)
        cv("dec2a", A["cat2"], 0, 256, A["d2a"], 0, 128, 2)
        cv("dec2b", A["d2a"], 0, 128, A["d2b"], 0, 128, 2)
        self._ck(L.sevp_nn_upsample(_p(A["d2b"]), 128, 0, _p(A["u1"]), 128, 0, 128, B, H // 2, W // 2, 0, self.sp), "up1")
        cv("up1", A["u1"], 0, 128, A["cat1"], 0, 128, 1)
        cv("dec1a", A["cat1"], 0, 128, A["d1a"], 0, 64, 1)
        cv("dec1b", A["d1a"], 0, 64, A["d1b"], 0, 64, 1)
        self._ck(L.sevp_nn_upsample(_p(A["d1b"]), 64, 0, _p(A["u0"]), 64, 0, 64, B, H, W, 0, self.sp), "up0")
        cv("up0", A["u0"], 0, 64, A["cat0"], 0, 64, 0)
        cv("dec0a", A["cat0"], 0, 64, A["d0a"], 0, 32, 0)
        cv("dec0b", A["d0a"], 0, 32, A["d0b"], 0, 32, 0)
        hw, hb = self.params["head"]
        self._ck(L.sevp_nn_head(_p(A["d0b"]), 32, 0, HEAD_C, _p(hw), _p(hb), _p(A["y"]), None, None, 0,
                                0, None, None, self.P[0], 0, self.sp), "head")
        return A["y"]

    # backward of one conv: dW (+ bias) and, if dsrc given, the data gradient
    def _conv_bwd(self, name, src, src_off, src_ld, gout, gout_off, gout_ld, out, out_off, out_ld,
                  dsrc, dsrc_off, dsrc_ld, lvl):
        _, ci, co = next(c for c in CONVS if c[0] == name)
        H, W = self.H >> lvl, self.W >> lvl
        L = lib()
        gw, gb = self.gw[name]
        # on the tcgen05 tensor cores: the ReLU-masked output gradient packed
        # once, the weight gradient as a pixel-contraction GEMM, the data
        # gradient as a forward conv with the tap-mirrored weights
        self._ck(L.sevp_nn_conv3x3_backward_tc(
            _p(src), src_ld, src_off, ci, _p(gout), gout_ld, gout_off, co, _p(out), out_ld, out_off,
            _p(self.wm16[name]), _p(self.gscratch), _p(gw), _p(gb),
            None if dsrc is None else _p(dsrc), dsrc_ld, dsrc_off, self.B, H, W, self.sp),
            name + " backward")

    def backward(self, target, valid=None):
        """MSE(y, target) -> parameter gradients in self.gw (zeroed first)."""
        A, G, L = self.A, self.G, lib()
        B, H, W = self.B, self.H, self.W
        for v in self.gw.values():
            v[0].zero_()
            v[1].zero_()
        self.loss.zero_()
        self._ck(L.sevp_nn_mse(_p(A["y"]), _p(target), _p(valid), _p(G["y"]), _p(self.loss), self.P[0],
                               1.0 / self.P[0], self.sp), "mse")
        hw, hb = self.params["head"]
        ghw, ghb = self.gw["head"]
        self._ck(L.sevp_nn_head(_p(A["d0b"]), 32, 0, HEAD_C, _p(hw), None, None, _p(G["y"]), _p(G["d0b"]),
                                32, 0, _p(ghw), _p(ghb), self.P[0], 1, self.sp), "head bwd")
        bw = self._conv_bwd
        bw("dec0b", A["d0a"], 0, 32, G["d0b"], 0, 32, A["d0b"], 0, 32, G["d0a"], 0, 32, 0)
        bw("dec0a", A["cat0"], 0, 64, G["d0a"], 0, 32, A["d0a"], 0, 32, G["cat0"], 0, 64, 0)
        bw("up0", A["u0"], 0, 64, G["cat0"], 0, 64, A["cat0"], 0, 64, G["u0"], 0, 64, 0)
        self._ck(L.sevp_nn_upsample(_p(G["u0"]), 64, 0, _p(G["d1b"]), 64, 0, 64, B, H, W, 1, self.sp), "up0 bwd")
        bw("dec1b", A["d1a"], 0, 64, G["d1b"], 0, 64, A["d1b"], 0, 64, G["d1a"], 0, 64, 1)
        bw("dec1a", A["cat1"], 0, 128, G["d1a"], 0, 64, A["d1a"], 0, 64, G["cat1"], 0, 128, 1)
        bw("up1", A["u1"], 0, 128, G["cat1"], 0, 128, A["cat1"], 0, 128, G["u1"], 0, 128, 1)
        self._ck(L.sevp_nn_upsample(_p(G["u1"]), 128, 0, _p(G["d2b"]), 128, 0, 128, B, H // 2, W // 2, 1, self.sp), "up1 bwd")
        bw("dec2b", A["d2a"], 0, 128, G["d2b"], 0, 128, A["d2b"], 0, 128, G["d2a"], 0, 128, 2)
        bw("dec2a", A["cat2"], 0, 256, G["d2a"], 0, 128, A["d2a"], 0, 128, G["cat2"], 0, 256, 2)
        bw("up2", A["u2"], 0, 256, G["cat2"], 0, 256, A["cat2"], 0, 256, G["u2"], 0, 256, 2)
        self._ck(L.sevp_nn_upsample(_p(G["u2"]), 256, 0, _p(G["b1"]), 256, 0, 256, B, H // 4, W // 4, 1, self.sp), "up2 bwd")
        bw("botb", A["b0"], 0, 256, G["b1"], 0, 256, A["b1"], 0, 256, G["b0"], 0, 256, 3)
        bw("bota", A["p2"], 0, 128, G["b0"], 0, 256, A["b0"], 0, 256, G["p2"], 0, 128, 3)
        # skip connection enc2b: concat-channel gradient + pooling gradient
        self._ck(L.sevp_nn_pool(_p(G["p2"]), 128, 0, _p(G["cat2"]), 256, 128, 128, B, H // 4, W // 4, 1, 1, self.sp), "pool2 bwd")
        bw("enc2b", A["e2a"], 0, 128, G["cat2"], 128, 256, A["cat2"], 128, 256, G["e2a"], 0, 128, 2)
        bw("enc2a", A["p1"], 0, 64, G["e2a"], 0, 128, A["e2a"], 0, 128, G["p1"], 0, 64, 2)
        self._ck(L.sevp_nn_pool(_p(G["p1"]), 64, 0, _p(G["cat1"]), 128, 64, 64, B, H // 2, W // 2, 1, 1, self.sp), "pool1 bwd")
        bw("enc1b", A["e1a"], 0, 64, G["cat1"], 64, 128, A["cat1"], 64, 128, G["e1a"], 0, 64, 1)
        bw("enc1a", A["p0"], 0, 32, G["e1a"], 0, 64, A["e1a"], 0, 64, G["p0"], 0, 32, 1)
        self._ck(L.sevp_nn_pool(_p(G["p0"]), 32, 0, _p(G["cat0"]), 64, 32, 32, B, H, W, 1, 1, self.sp), "pool0 bwd")
        bw("enc0b", A["e0a"], 0, 32, G["cat0"], 32, 64, A["cat0"], 32, 64, G["e0a"], 0, 32, 0)
        bw("enc0a", A["x"], 0, IN_C, G["e0a"], 0, 32, A["e0a"], 0, 32, None, 0, 0, 0)

    def adam_step(self, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8, wd=0.0):
        L = lib()
        self.step_count += 1
        for name, (w, b) in self.params.items():
            gw, gb = self.gw[name]
            mw, mb = self.m[name]
            vw, vb = self.v[name]
            if name == "enc0a":
                gw[:, 3:, :].zero_()  # padded input channels stay zero
            w16 = self.w16[name] if name in self.w16 else None
            self._ck(L.sevp_nn_adam(_p(w), _p(gw), _p(mw), _p(vw), _p(w16), None, w.numel(), lr, b1, b2,
                                    eps, self.step_count, wd, self.sp), "adam w")
            self._ck(L.sevp_nn_adam(_p(b), _p(gb), _p(mb), _p(vb), None, None, b.numel(), lr, b1, b2, eps,
                                    self.step_count, 0.0, self.sp), "adam b")
        for name, ci, co in CONVS:
            self._ck(lib().sevp_nn_weight_transpose(_p(self.w16[name]), _p(self.wt16[name]), ci, co,
                                                    self.sp), "transpose")
            # the data gradient's tap-mirrored copy follows the new weights
            self._ck(lib().sevp_nn_weight_mirror(_p(self.w16[name]), _p(self.wm16[name]), ci, co,
                                                 self.sp), "mirror")

    # ---------------------------------------------------------- weights io
    def state(self) -> dict:
        return {f"{n}.{k}": v[k].detach().cpu().numpy() for n, v in self.params.items() for k in (0, 1)}

    def load_state(self, st: dict):
        for n, v in self.params.items():
            for k in (0, 1):
                v[k].copy_(self.torch.from_numpy(np.asarray(st[f"{n}.{k}"], np.float32)))
        self.sync_weights()

    def flops_forward(self) -> float:
        f = 0.0
        lvl = {"enc0a": 0, "enc0b": 0, "enc1a": 1, "enc1b": 1, "enc2a": 2, "enc2b": 2, "bota": 3,
               "botb": 3, "up2": 2, "dec2a": 2, "dec2b": 2, "up1": 1, "dec1a": 1, "dec1b": 1,
               "up0": 0, "dec0a": 0, "dec0b": 0}
        for name, ci, co in CONVS:
            f += 2.0 * 9 * ci * co * self.P[lvl[name]]
        return f + 2.0 * HEAD_C * self.P[0]
