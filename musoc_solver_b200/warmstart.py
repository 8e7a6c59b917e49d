"""Learned warm start for a time sequence of barotropic solves.

For step n the guess is

    x = e + m + s_m * y,   e = 2 eta_{n-1} - eta_{n-2},   m = M^{-1} (b_n - A e),

where M^{-1} is one application of the tile-SEVP preconditioner and y is the
U-Net's output for the three normalised input channels
(b_n - A e) / s_r, m / s_m, (eta_{n-1} - eta_{n-2}) / s_d
(s_* = RMS over the field).  The network therefore learns the part of the
exact correction A^{-1} (b_n - A e) that one block-Jacobi tile solve misses
(the coupling across tile edges).  It is trained on solutions the solver
itself produces; the solve from the guess to 1e-12 stays the judge.

Everything runs on the GPU in ``libsevp_b200.so``: the feature, target and
combine kernels, the U-Net forward/backward kernels, Adam.  Inference is
captured in a CUDA graph and replayed from the solver's warm-start hook.
"""
from __future__ import annotations

import ctypes as C
import time

import numpy as np

from . import native as N
from .unet import UNet, lib as nnlib

COARSE = (1, 2, 4, 8, 16)


def net_grid(nx: int, ny: int, coarse: int):
    """(H, W) of the network for a solver grid averaged over coarse x coarse
    cells, rounded up to multiples of 8."""
    if coarse not in COARSE or nx % coarse or ny % coarse:
        raise ValueError("coarse must be 1, 2, 4, 8 or 16 and divide the grid")
    r8 = lambda v: (v + 7) // 8 * 8
    return r8(ny // coarse), r8(nx // coarse)


WARMSTART_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                           C.c_int, C.c_int, C.c_void_p)


class LearnedWarmStart:
    """Binds a U-Net to a solver context of the same grid."""

    def __init__(self, solver, unet: UNet, use_graph: bool = True):
        import torch

        self.torch = torch
        self.solver = solver
        self.net = unet
        # the network grid: the solver grid averaged over coarse x coarse
        # cells, padded to multiples of 8
        self.coarse = next((c for c in COARSE if solver.nx % c == 0 and solver.ny % c == 0
                            and net_grid(solver.nx, solver.ny, c) == (unet.H, unet.W)), None)
        if self.coarse is None:
            raise ValueError("network grid does not match the solver grid at coarse 1, 2, 4 or 8")
        self._g = (self.coarse, unet.W, unet.H)
        n = unet.H * unet.W
        dev = solver.device
        self.e = torch.zeros((solver.ny, solver.nx), dtype=torch.float64, device=dev)
        self.m = torch.zeros_like(self.e)
        self.d = torch.zeros_like(self.e)
        self.scales = torch.ones(4, dtype=torch.float32, device=dev)
        self.target = torch.zeros(n, dtype=torch.float32, device=dev)
        self.graph = None
        self.use_graph = use_graph
        self._cb = None
        nnlib()

    # ---------------------------------------------------------------- core
    def features(self, eta1, eta2, b):
        s = nnlib().sevp_nn_features(self.solver.h, C.c_void_p(int(eta1)), C.c_void_p(int(eta2)),
                                     C.c_void_p(int(b)), C.c_void_p(self.e.data_ptr()),
                                     C.c_void_p(self.m.data_ptr()), C.c_void_p(self.d.data_ptr()),
                                     C.c_void_p(self.net.A["x"].data_ptr()),
                                     C.c_void_p(self.scales.data_ptr()), *self._g)
        N.check(s, "sevp_nn_features")

    def _forward(self):
        if self.use_graph:
            if self.graph is None:
                torch = self.torch
                self.net.forward()  # warm-up outside the capture
                torch.cuda.synchronize()
                g = torch.cuda.CUDAGraph()
                # capture on a side stream (the legacy default stream cannot
                # be captured); the replay runs on the current stream
                cs = torch.cuda.Stream(device=self.solver.device)
                cs.wait_stream(torch.cuda.current_stream(self.solver.device))
                old = self.net.sp
                self.net.sp = C.c_void_p(cs.cuda_stream)
                try:
                    with torch.cuda.graph(g, stream=cs):
                        self.net.forward()
                finally:
                    self.net.sp = old
                self.graph = g
            self.graph.replay()
        else:
            self.net.forward()

    def predict(self, eta1, eta2, b, x):
        """x <- guess (raw device pointers or tensors)."""
        ptr = lambda t: t.data_ptr() if hasattr(t, "data_ptr") else int(t)
        self.features(ptr(eta1), ptr(eta2), ptr(b))
        self._forward()
        s = nnlib().sevp_nn_combine(self.solver.h, C.c_void_p(self.e.data_ptr()),
                                    C.c_void_p(self.m.data_ptr()),
                                    C.c_void_p(self.net.A["y"].data_ptr()),
                                    C.c_void_p(self.scales.data_ptr()), C.c_void_p(ptr(x)),
                                    *self._g)
        N.check(s, "sevp_nn_combine")

    def attach(self, solver=None):
        """Registers the network as the solver's SEVP_GUESS_LEARNED hook."""
        solver = solver or self.solver

        def cb(user, eta1, eta2, b, x, nx, ny, stream):
            try:
                self.predict(eta1, eta2, b, x)
                return 0
            except Exception:
                return N.SEVP_CUDA_ERROR

        self._cb = WARMSTART_FN(cb)
        # launches per call: 6 feature kernels + network (graph) + combine
        per_call = 7 + 20
        N.check(N.lib().sevp_set_warmstart(solver.h, C.cast(self._cb, C.c_void_p), None, per_call),
                "sevp_set_warmstart")

    def close(self):
        if self._cb is not None:
            N.lib().sevp_set_warmstart(self.solver.h, None, None, 0)
            self._cb = None
        self.graph = None

    # ------------------------------------------------------------ training
    def train_step(self, eta1, eta2, b, eta, lr=1e-3):
        """One Adam step on the sample (eta_{n-1}, eta_{n-2}, b_n) -> eta_n."""
        self.features(eta1.data_ptr(), eta2.data_ptr(), b.data_ptr())
        s = nnlib().sevp_nn_target(self.solver.h, C.c_void_p(eta.data_ptr()),
                                   C.c_void_p(self.e.data_ptr()), C.c_void_p(self.m.data_ptr()),
                                   C.c_void_p(self.scales.data_ptr()),
                                   C.c_void_p(self.target.data_ptr()), *self._g)
        N.check(s, "sevp_nn_target")
        self.net.forward()
        self.net.backward(self.target)
        self.net.adam_step(lr=lr)
        return self.net.loss

    def save(self, path):
        st = self.net.state()
        np.savez(path, **st)

    @classmethod
    def load(cls, path, solver, coarse=1):
        """Inference-only network for the solver's grid from saved weights."""
        st = dict(np.load(path))
        H, W = net_grid(solver.nx, solver.ny, coarse)
        net = UNet(H, W, device=solver.device, train=False, stream=solver.stream)
        net.load_state(st)
        return cls(solver, net)

    @classmethod
    def create(cls, solver, seed=0, train=True, coarse=1):
        """A fresh network on the solver grid averaged over coarse x coarse
        cells (coarse = 1, 2, 4 or 8)."""
        H, W = net_grid(solver.nx, solver.ny, coarse)
        net = UNet(H, W, device=solver.device, train=train, seed=seed, stream=solver.stream)
        return cls(solver, net, use_graph=not train)

    def inference_copy(self):
        """A graph-captured inference-only warm start with the trained weights."""
        net = UNet(self.net.H, self.net.W, device=self.solver.device, train=False,
                   stream=self.solver.stream)
        net.load_state(self.net.state())
        return LearnedWarmStart(self.solver, net, use_graph=True)


def solve_sequence(solver, rhs, tol=1e-12):
    """FP64 solves of a right-hand-side sequence (device tensors), each from
    the linear extrapolation of the two previous solutions."""
    import torch

    etas = []
    for n, b in enumerate(rhs):
        x = torch.zeros_like(b)
        if n >= 2:
            solver.solve_step(b, etas[n - 1], etas[n - 2], x, guess=N.GUESS_LINEAR, precision=0, tol=tol)
        elif n == 1:
            solver.solve_step(b, etas[0], None, x, guess=N.GUESS_PREVIOUS, precision=0, tol=tol)
        else:
            solver.solve(b, x=None, precision=0, tol=tol)
            x.copy_(solver.solve(b, precision=0, tol=tol)[0])
        etas.append(x)
    return etas


def train(warm: LearnedWarmStart, etas, rhs, train_idx, epochs=4, lr=1e-3, lr_final=1e-4, seed=0,
          log=None):
    """Adam over the training steps (full fields, batch 1), cosine-decayed lr."""
    rng = np.random.default_rng(seed)
    total = epochs * len(train_idx)
    k = 0
    losses = []
    t0 = time.time()
    for ep in range(epochs):
        order = rng.permutation(train_idx)
        for n in order:
            frac = k / max(total - 1, 1)
            lr_k = lr_final + 0.5 * (lr - lr_final) * (1 + np.cos(np.pi * frac))
            loss = warm.train_step(etas[n - 1], etas[n - 2], rhs[n], etas[n], lr=lr_k)
            k += 1
            if k % 50 == 0 or k == total:
                lv = float(loss.item())
                losses.append((k, lv))
                if log:
                    log(f"step {k}/{total} loss {lv:.4e} ({time.time() - t0:.1f}s)")
    return losses


def evaluate(solver, warm, etas, rhs, idx, precision=1, tol=1e-12):
    """Iterations and device time to tol from each guess."""
    import torch

    res = {}
    x = torch.zeros_like(etas[0])
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for name, mode in (("zero", N.GUESS_ZERO), ("previous", N.GUESS_PREVIOUS),
                       ("linear", N.GUESS_LINEAR), ("learned", N.GUESS_LEARNED)):
        if mode == N.GUESS_LEARNED and warm is None:
            continue
        its, ms, err = [], [], []
        for n in idx:
            x.zero_()
            e0.record(solver.stream)
            _, r = solver.solve_step(rhs[n], etas[n - 1], etas[n - 2], x, guess=mode,
                                     precision=precision, tol=tol)
            e1.record(solver.stream)
            e1.synchronize()
            its.append(r.iterations)
            ms.append(e0.elapsed_time(e1))  # guess + solve
            err.append(float((x - etas[n]).abs().max() / etas[n].abs().max()))
        res[name] = {"mean_iterations": float(np.mean(its)), "mean_ms": float(np.mean(ms)),
                     "max_rel_err_vs_fp64": float(np.max(err))}
    return res
