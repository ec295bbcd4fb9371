"""The closure CNN: six 3x3 convolutions (1 -> 64 -> 64 -> 64 -> 64 -> 64 -> 1)
with GELU between them and circular padding, BF16 activations and weights
on the tensor cores with FP32 accumulation, FP32 master weights and Adam.

All compute runs in the library's kernels (include/sqg_closure.h); torch
holds the buffers.  Layer l in 2..5 is the tcgen05 convolution; layers 1 and
6 (one channel in / out) run on CUDA cores.
"""

from __future__ import annotations

import math

import numpy as np
import torch

from .. import _lib
from . import _ops

C64 = 64
_NRED = 296 * (9 * 64 + 64)


def _sp():
    return torch.cuda.current_stream().cuda_stream


def _chk(rc):
    if rc != 0:
        L = _lib.load()
        raise RuntimeError(L.closure_ops_last_error_string().decode() or L.closure_last_error_string().decode())


class ClosureCNN:
    """Parameters live in one flat FP32 vector (one Adam launch updates all)."""

    SHAPES = [("w1", (9, 64)), ("b1", (64,))] + [
        x for l in range(2, 6) for x in ((f"w{l}", (9, 64, 64)), (f"b{l}", (64,)))
    ] + [("w6", (9, 64)), ("b6", (1,))]

    def __init__(self, H: int = 256, W: int = 256, max_batch: int = 8, seed: int = 0, device="cuda"):
        assert W % 128 == 0, "W must be a multiple of 128"
        self.H, self.W, self.maxB, self.dev = H, W, max_batch, device
        n = sum(int(np.prod(s)) for _, s in self.SHAPES)
        self.flat = torch.zeros(n, dtype=torch.float32, device=device)
        self.grad = torch.zeros_like(self.flat)
        self.m = torch.zeros_like(self.flat)
        self.v = torch.zeros_like(self.flat)
        self.p, self.g = {}, {}
        o = 0
        for name, shp in self.SHAPES:
            k = int(np.prod(shp))
            self.p[name] = self.flat[o:o + k].view(shp)
            self.g[name] = self.grad[o:o + k].view(shp)
            o += k
        rng = np.random.default_rng(seed)
        for name, shp in self.SHAPES:
            if name.startswith("w"):
                fan_in = 9 if name == "w1" else 9 * 64
                self.p[name].copy_(torch.as_tensor(rng.standard_normal(shp) * math.sqrt(2.0 / fan_in)))
        self.step_count = 0
        self.wf = {l: torch.empty(9, 64, 64, dtype=torch.bfloat16, device=device) for l in range(2, 6)}
        self.wb = {l: torch.empty(9, 64, 64, dtype=torch.bfloat16, device=device) for l in range(2, 6)}
        B, Hp, Wp = max_batch, H + 2, W + 2
        self.a = {l: torch.zeros(B, Hp, Wp, 64, dtype=torch.bfloat16, device=device) for l in range(1, 6)}
        self.z = {l: torch.zeros(B, H, W, 64, dtype=torch.bfloat16, device=device) for l in range(1, 6)}
        self.gz = [torch.zeros(B, Hp, Wp, 64, dtype=torch.bfloat16, device=device) for _ in range(2)]
        self.y = torch.zeros(B, H, W, dtype=torch.float32, device=device)
        self.gy = torch.zeros_like(self.y)
        self.red = torch.empty(_NRED, dtype=torch.float32, device=device)
        self.redout = torch.empty(9 * 64 + 64, dtype=torch.float32, device=device)
        self.wpart = torch.empty(148 * 5 * 128 * 64, dtype=torch.float32, device=device)
        self.loss_part = torch.empty(296, dtype=torch.float32, device=device)
        self.err = torch.zeros(1, dtype=torch.int32, device=device)
        self.refresh()

    def refresh(self):
        """BF16 tensor-core copies of the middle-layer weights."""
        L = _lib.load()
        for l in range(2, 6):
            _chk(L.closure_weights_bf16(self.p[f"w{l}"].data_ptr(), self.wf[l].data_ptr(), self.wb[l].data_ptr(), _sp()))

    # ---- forward / backward ----
    def forward(self, x: torch.Tensor, in_scale: float = 1.0, out_scale: float = 1.0) -> torch.Tensor:
        """x: FP32 [B, H, W] -> y: FP32 [B, H, W] (a view of an internal buffer).

        ``in_scale`` / ``out_scale`` multiply the input and the output (a data
        normalisation folded into the first and last layers)."""
        L = _lib.load()
        B = x.shape[0]
        assert x.shape[1:] == (self.H, self.W) and B <= self.maxB and x.dtype == torch.float32
        x = x.contiguous()
        H, W = self.H, self.W
        a = {l: self.a[l][:B] for l in self.a}
        z = {l: self.z[l][:B] for l in self.z}
        _chk(L.closure_conv_in(B, H, W, in_scale, x.data_ptr(), self.p["w1"].data_ptr(), self.p["b1"].data_ptr(),
                               z[1].data_ptr(), a[1].data_ptr(), _sp()))
        for l in range(2, 6):
            _ops.conv64(a[l - 1], self.wf[l], _ops.CLOSURE_EPI_FWD, bias=self.p[f"b{l}"], out_pad=a[l], out_z=z[l],
                        err=self.err)
        y = self.y[:B]
        _chk(L.closure_conv_out(B, H, W, out_scale, a[5].data_ptr(), self.p["w6"].data_ptr(), self.p["b6"].data_ptr(),
                                y.data_ptr(), _sp()))
        return y

    def backward(self, x: torch.Tensor, gy: torch.Tensor) -> None:
        """Gradients of all parameters into self.grad for dL/dy = gy."""
        L = _lib.load()
        B = x.shape[0]
        H, W = self.H, self.W
        x = x.contiguous()
        gy = gy.contiguous()
        a = {l: self.a[l][:B] for l in self.a}
        z = {l: self.z[l][:B] for l in self.z}
        gz = [t[:B] for t in self.gz]
        _chk(L.closure_small_grad(0, B, H, W, gy.data_ptr(), a[5].data_ptr(), None, None, self.red.data_ptr(),
                                  self.redout.data_ptr(), _sp()))
        self.g["w6"].copy_(self.redout[:576].view(9, 64))
        self.g["b6"].copy_(self.redout[576:577])
        cur = 0
        _chk(L.closure_conv_out_dgrad(B, H, W, gy.data_ptr(), self.p["w6"].data_ptr(), z[5].data_ptr(),
                                      gz[cur].data_ptr(), _sp()))
        for l in range(5, 1, -1):
            dw, _ = _ops.wgrad64(a[l - 1], gz[cur], nparts=148, err=self.err, partials=self.wpart)
            self.g[f"w{l}"].copy_(dw)
            _chk(L.closure_small_grad(2, B, H, W, None, None, None, gz[cur].data_ptr(), self.red.data_ptr(),
                                      self.redout.data_ptr(), _sp()))
            self.g[f"b{l}"].copy_(self.redout[576:640])
            _ops.conv64(gz[cur], self.wb[l], _ops.CLOSURE_EPI_DGRAD, zprev=z[l - 1], out_pad=gz[1 - cur], err=self.err)
            cur = 1 - cur
        _chk(L.closure_small_grad(1, B, H, W, None, None, x.data_ptr(), gz[cur].data_ptr(), self.red.data_ptr(),
                                  self.redout.data_ptr(), _sp()))
        self.g["w1"].copy_(self.redout[:576].view(9, 64))
        self.g["b1"].copy_(self.redout[576:640])

    def mse(self, y: torch.Tensor, t: torch.Tensor) -> torch.Tensor:
        """Loss (device scalar) and dL/dy into self.gy."""
        L = _lib.load()
        B = y.shape[0]
        gy = self.gy[:B]
        _chk(L.closure_mse(y.numel(), y.data_ptr(), t.contiguous().data_ptr(), gy.data_ptr(),
                           self.loss_part.data_ptr(), _sp()))
        return self.loss_part.sum() / y.numel()

    def train_step(self, x, t, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
        y = self.forward(x)
        loss = self.mse(y, t)
        self.backward(x, self.gy[: x.shape[0]])
        self.step_count += 1
        _chk(_lib.load().closure_adam(self.flat.numel(), self.flat.data_ptr(), self.grad.data_ptr(), self.m.data_ptr(),
                                      self.v.data_ptr(), lr, b1, b2, eps, self.step_count, _sp()))
        self.refresh()
        return loss

    def errors(self) -> int:
        return int(self.err.item())

    def state_dict(self):
        return {k: v.detach().cpu().clone() for k, v in self.p.items()}

    def load_state_dict(self, d):
        for k, v in d.items():
            self.p[k].copy_(v.to(self.dev))
        self.refresh()


def _main(argv=None) -> int:
    """Time the network: python -m pygsquig_b200.closure.cnn [--batch B] [--reps R]
    (CUDA events; forward at batch 1 and a training step at batch B)."""
    import argparse
    import json

    ap = argparse.ArgumentParser()
    ap.add_argument("--size", type=int, default=256)
    ap.add_argument("--batch", type=int, default=16)
    ap.add_argument("--reps", type=int, default=20)
    a = ap.parse_args(argv)
    from ..build import build

    build()
    net = ClosureCNN(a.size, a.size, max_batch=a.batch)
    x1 = torch.randn(1, a.size, a.size, device="cuda")
    xb = torch.randn(a.batch, a.size, a.size, device="cuda")
    for _ in range(3):
        net.forward(x1)
        net.train_step(xb, xb, lr=0.0)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    ev[0].record()
    for _ in range(a.reps):
        net.forward(x1)
    ev[1].record()
    for _ in range(a.reps):
        net.train_step(xb, xb, lr=0.0)
    ev[2].record()
    torch.cuda.synchronize()
    if net.errors():
        raise RuntimeError("closure kernels reported a timed-out wait")
    fwd = ev[0].elapsed_time(ev[1]) / a.reps
    trn = ev[1].elapsed_time(ev[2]) / a.reps
    flop = 4 * 2 * 9 * 64 * 64 * a.size * a.size
    print(json.dumps({"forward_ms_batch1": fwd, "train_step_ms": trn, "batch": a.batch,
                      "forward_tensor_tflops": flop / fwd * 1e-9,
                      "train_tensor_tflops": 3 * flop * a.batch / trn * 1e-9}))
    return 0


if __name__ == "__main__":
    raise SystemExit(_main())
