"""ctypes binding of the closure kernels (include/sqg_closure.h)."""

from __future__ import annotations

import ctypes as C

import torch

from .. import _lib

CLOSURE_EPI_FWD, CLOSURE_EPI_DGRAD, CLOSURE_EPI_LIN = 0, 1, 2

def lib():
    return _lib.load()


def _p(t):
    return None if t is None else t.data_ptr()


def check(rc):
    if rc != 0:
        raise RuntimeError(lib().closure_last_error_string().decode())


def conv64(act_pad: torch.Tensor, weights: torch.Tensor, mode: int, bias=None, zprev=None, out_pad=None, out_z=None,
           out_f32=None, err=None, grid: int = 0):
    """3x3 conv 64->64 on the tensor cores.  act_pad: BF16 [B, H+2, W+2, 64];
    weights: BF16 [9, 64, 64] (tap, out, in)."""
    B, Hp, Wp, Cc = act_pad.shape
    assert Cc == 64 and act_pad.dtype == torch.bfloat16 and weights.dtype == torch.bfloat16
    if err is None:
        err = torch.zeros(1, dtype=torch.int32, device=act_pad.device)
    check(lib().closure_conv64(B, Hp - 2, Wp - 2, mode, _p(act_pad), _p(weights), _p(bias), _p(zprev), _p(out_pad),
                               _p(out_z), _p(out_f32), _p(err), grid, torch.cuda.current_stream().cuda_stream))
    return err


def wgrad64(act_pad: torch.Tensor, grad_pad: torch.Tensor, nparts: int = 148, err=None, partials=None):
    """dW[t, co, ci] = sum_p act[p + off_t, ci] grad[p, co] (FP32 [9, 64, 64])."""
    B, Hp, Wp, Cc = act_pad.shape
    assert grad_pad.shape == act_pad.shape and Cc == 64
    if err is None:
        err = torch.zeros(1, dtype=torch.int32, device=act_pad.device)
    if partials is None:
        partials = torch.empty(nparts * 5 * 128 * 64, dtype=torch.float32, device=act_pad.device)
    dw = torch.empty(9, 64, 64, dtype=torch.float32, device=act_pad.device)
    check(lib().closure_wgrad64(B, Hp - 2, Wp - 2, _p(act_pad), _p(grad_pad), _p(partials), nparts, _p(dw), _p(err),
                                torch.cuda.current_stream().cuda_stream))
    return dw, err
