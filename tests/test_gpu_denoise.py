"""The denoiser's tcgen05 convolution kernels against PyTorch's fp32 convolution on the same
bf16-rounded operands: forward (bias, ReLU, channel slices, bf16 and fp32 outputs, N tails of
every tile width), weight gradient and data gradient. Tolerance: fp32 accumulation order only
(relative 2e-3 of the output's scale), or one bf16 rounding for bf16 outputs."""
import numpy as np
import pytest

from conftest import load_package

pytestmark = pytest.mark.gpu
PKG = load_package()


def _dn():
    import importlib
    return importlib.import_module(PKG.__name__ + ".denoise")


def _setup(B, H, W, ldx, xoff, cin, cout, seed):
    import torch
    g = torch.Generator().manual_seed(seed)
    dn = _dn()
    x = torch.zeros(B, H, W, ldx)
    x[..., xoff:xoff + cin] = torch.randn(B, H, W, cin, generator=g)
    kp = dn.kp_of(cin)
    w = torch.zeros(cout, kp)
    w[:, :9 * cin] = torch.randn(cout, 9 * cin, generator=g) * 0.2
    bias = torch.randn(cout, generator=g)
    xb = x.to(torch.bfloat16)
    wb = w.to(torch.bfloat16)
    w_t = wb.float()[:, :9 * cin].reshape(cout, 3, 3, cin).permute(0, 3, 1, 2).contiguous()
    x_t = xb.float()[..., xoff:xoff + cin].permute(0, 3, 1, 2).contiguous()
    return dn, xb.cuda(), wb.cuda(), bias.cuda(), x_t, w_t, bias


@pytest.mark.parametrize("cout", [3, 16, 40, 128, 200])
def test_conv_forward_fp32(cout):
    import torch
    import torch.nn.functional as F
    B, H, W, cin = 2, 19, 23, 16
    dn, xb, wb, bias, x_t, w_t, bias_c = _setup(B, H, W, 24, 8, cin, cout, cout)
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    out = torch.full((B, H, W, cout + 5), -7.0, device="cuda")
    dn.conv_fwd(xb, cin, wb, cout, bias, out, xoff=8, ooff=5, err=err)
    torch.cuda.synchronize()
    ref = F.conv2d(x_t, w_t, bias_c, padding=1).permute(0, 2, 3, 1)
    got = out[..., 5:].cpu()
    scale = ref.abs().max().item()
    assert (got - ref).abs().max().item() <= 2e-3 * scale, (got - ref).abs().max().item()
    assert torch.all(out[..., :5] == -7.0)
    assert int(err.item()) == 0


def test_conv_forward_bf16_relu():
    import torch
    import torch.nn.functional as F
    B, H, W, cin, cout = 3, 16, 16, 32, 64
    dn, xb, wb, bias, x_t, w_t, bias_c = _setup(B, H, W, 32, 0, cin, cout, 7)
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    out = torch.zeros((B, H, W, cout), dtype=torch.bfloat16, device="cuda")
    dn.conv_fwd(xb, cin, wb, cout, bias, out, relu=True, err=err)
    torch.cuda.synchronize()
    ref = F.relu(F.conv2d(x_t, w_t, bias_c, padding=1)).permute(0, 2, 3, 1)
    got = out.float().cpu()
    assert torch.allclose(got, ref, rtol=1.0 / 128, atol=2e-3 * ref.abs().max().item())
    assert int(err.item()) == 0


@pytest.mark.parametrize("cin,cout", [(8, 32), (32, 64), (64, 3)])
def test_conv_weight_and_data_gradient(cin, cout):
    import torch
    import torch.nn.grad as G
    B, H, W = 2, 24, 20
    dn, xb, wb, bias, x_t, w_t, _ = _setup(B, H, W, cin, 0, cin, cout, cin + cout)
    g = torch.Generator().manual_seed(11)
    coutp = (cout + 7) // 8 * 8
    dy = torch.zeros(B, H, W, coutp)
    dy[..., :cout] = torch.randn(B, H, W, cout, generator=g)
    dyb = dy.to(torch.bfloat16)
    dy_t = dyb.float()[..., :cout].permute(0, 3, 1, 2).contiguous()
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    # weight gradient
    dw = torch.zeros(cout, wb.shape[1], device="cuda")
    dn.conv_dw(dyb.cuda(), xb, cin, cout, dw, err=err)
    torch.cuda.synchronize()
    ref_w = G.conv2d_weight(x_t, w_t.shape, dy_t, padding=1)  # (cout, cin, 3, 3)
    got_w = dw.cpu()[:, :9 * cin].reshape(cout, 3, 3, cin).permute(0, 3, 1, 2)
    assert (got_w - ref_w).abs().max().item() <= 2e-3 * ref_w.abs().max().item()
    assert torch.all(dw.cpu()[:, 9 * cin:] == 0)
    # data gradient: the forward convolution of dy with the flipped weights
    kp2 = dn.kp_of(coutp)
    wf = torch.zeros(cin, kp2, dtype=torch.bfloat16, device="cuda")
    dn.flip(wb, cout, cin, wf, coutp)
    dx = torch.zeros(B, H, W, cin, device="cuda")
    dn.conv_fwd(dyb.cuda(), coutp, wf, cin, None, dx, err=err)
    torch.cuda.synchronize()
    ref_x = G.conv2d_input(x_t.shape, w_t, dy_t, padding=1).permute(0, 2, 3, 1)
    assert (dx.cpu() - ref_x).abs().max().item() <= 2e-3 * ref_x.abs().max().item()
    assert int(err.item()) == 0
