"""tcgen05 3x3 convolution (64 -> 64 channels, circular padding) against
torch.nn.functional.conv2d in float32 on the same BF16 inputs."""

import pytest
import torch
import torch.nn.functional as F

pytestmark = pytest.mark.gpu


def halo(x):  # [B, H, W, C] -> [B, H+2, W+2, C] circular
    return F.pad(x.permute(0, 3, 1, 2), (1, 1, 1, 1), mode="circular").permute(0, 2, 3, 1).contiguous()


def ref_conv(x_bhwc, w_t_oi, bias):
    # w_t_oi: [9, out, in] with tap t = 3 (dy+1) + (dx+1) -> torch weight [out, in, 3, 3]
    w = w_t_oi.reshape(3, 3, 64, 64).permute(2, 3, 0, 1)
    xp = F.pad(x_bhwc.permute(0, 3, 1, 2), (1, 1, 1, 1), mode="circular")
    return F.conv2d(xp, w, bias).permute(0, 2, 3, 1)


@pytest.mark.parametrize("B,H,W", [(1, 4, 128), (2, 8, 256)])
def test_conv64_forward_and_dgrad(B, H, W):
    from pygsquig_b200.build import build

    build()
    from pygsquig_b200.closure import _ops

    torch.manual_seed(0)
    dev = "cuda"
    x = torch.randn(B, H, W, 64, device=dev).to(torch.bfloat16)
    w = (torch.randn(9, 64, 64, device=dev) * 0.05).to(torch.bfloat16)
    b = torch.randn(64, device=dev) * 0.1
    xp = halo(x)
    # LIN: plain conv + bias in FP32
    out = torch.empty(B, H, W, 64, device=dev)
    err = _ops.conv64(xp, w, _ops.CLOSURE_EPI_LIN, bias=b, out_f32=out)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    ref = ref_conv(x.float(), w.float(), b)
    e = (out - ref).abs().max().item() / ref.abs().max().item()
    assert e < 1e-5, e
    # FWD: z (BF16) and gelu(z) with halo
    zo = torch.empty(B, H, W, 64, device=dev, dtype=torch.bfloat16)
    ao = torch.zeros(B, H + 2, W + 2, 64, device=dev, dtype=torch.bfloat16)
    _ops.conv64(xp, w, _ops.CLOSURE_EPI_FWD, bias=b, out_pad=ao, out_z=zo, err=err)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    zr = ref.to(torch.bfloat16)
    assert (zo.float() - zr.float()).abs().max().item() <= 0.02 * ref.abs().max().item()
    gz = F.gelu(zo.float()).to(torch.bfloat16)
    assert torch.allclose(ao.float(), halo(gz).float(), atol=2e-2, rtol=2e-2)
    # DGRAD: conv * gelu'(zprev)
    zprev = torch.randn(B, H, W, 64, device=dev).to(torch.bfloat16)
    go = torch.zeros_like(ao)
    _ops.conv64(xp, w, _ops.CLOSURE_EPI_DGRAD, zprev=zprev, out_pad=go, err=err)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    zf = zprev.float()
    gprime = 0.5 * (1 + torch.erf(zf / 2**0.5)) + zf * torch.exp(-0.5 * zf * zf) / (2 * torch.pi) ** 0.5
    gr = (ref_conv(x.float(), w.float(), None) * gprime).to(torch.bfloat16)
    assert torch.allclose(go.float(), halo(gr).float(), atol=2e-2 * gr.float().abs().max().item(), rtol=2e-2)


@pytest.mark.parametrize("B,H,W", [(1, 4, 128), (2, 8, 256)])
def test_wgrad64(B, H, W):
    from pygsquig_b200.build import build

    build()
    from pygsquig_b200.closure import _ops

    torch.manual_seed(1)
    dev = "cuda"
    a = torch.randn(B, H, W, 64, device=dev).to(torch.bfloat16)
    g = torch.randn(B, H, W, 64, device=dev).to(torch.bfloat16)
    dw, err = _ops.wgrad64(halo(a), halo(g), nparts=7)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    # reference: dW[t, co, ci] = sum_p a[p + off_t, ci] g[p, co]
    ap = halo(a).float()
    ref = torch.empty(9, 64, 64, device=dev)
    for t in range(9):
        dy, dx = t // 3 - 1, t % 3 - 1
        sh = ap[:, 1 + dy:1 + dy + H, 1 + dx:1 + dx + W, :]
        ref[t] = torch.einsum("bhwo,bhwi->oi", g.float(), sh)
    e = (dw - ref).abs().max().item() / ref.abs().max().item()
    assert e < 1e-4, e
