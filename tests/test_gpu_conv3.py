"""The TMA-staged 3x3 convolution (gpsb_dn_conv3, csrc/conv3x3.cu) on chunk-planar activations
against PyTorch's fp32 convolution of the same bf16-rounded operands, for every output width the
kernel instantiates (16 .. 192 channels), the input widths of the U-Net and of its data gradients
(8 .. 192), images whose width is not a multiple of the 126-pixel segment and whose height is not a
multiple of the row block, batches, channel slices of wider tensors (input offset, output offset),
bf16 (chunk-planar) and fp32 (pixel-major) outputs, bias and ReLU. Tolerance: fp32 accumulation
order (2e-3 of the output's scale), or one bf16 rounding for bf16 outputs. The whole U-Net on
these kernels is compared with the float64 oracle's forward pass."""
import numpy as np
import pytest

from conftest import load_package

pytestmark = pytest.mark.gpu
PKG = load_package()
torch = pytest.importorskip("torch")
F = torch.nn.functional


def _dn():
    import importlib
    return importlib.import_module(PKG.__name__ + ".denoise")


CASES = [
    # B, H, W, ldx, xoff, cin, cout, ldo, ooff, fp32 out, relu
    (1, 9, 200, 8, 0, 8, 32, 32, 0, False, True),        # c1a: one input chunk (the second reads as zeros)
    (2, 11, 130, 32, 0, 32, 32, 96, 64, False, True),    # c1b into the concatenation slice
    (1, 7, 64, 32, 0, 32, 64, 64, 0, False, True),       # c2a
    (2, 6, 96, 64, 0, 64, 128, 128, 0, False, True),     # c3a
    (1, 5, 40, 128, 0, 128, 128, 128, 0, False, False),  # c3b
    (1, 6, 150, 192, 0, 192, 64, 64, 0, False, True),    # c4a
    (2, 13, 256, 96, 0, 96, 32, 32, 0, False, True),     # c5a
    (1, 10, 140, 32, 0, 32, 3, 3, 0, True, False),       # c6: 3 outputs, fp32, scalar stores
    (1, 6, 70, 32, 0, 32, 20, 24, 0, False, False),      # bf16 output with a partial chunk (scalar stores)
    (1, 9, 300, 40, 8, 24, 96, 96, 0, True, False),      # data gradient of c5a (96 out), offset input
    (1, 4, 129, 64, 0, 64, 192, 200, 8, True, False),    # data gradient of c4a (192 out), offset output
    (3, 8, 128, 8, 0, 8, 16, 16, 0, True, False),        # N = 16 with 16 outputs
    (1, 9, 126, 32, 0, 32, 32, 32, 0, False, True),      # exactly one 126-pixel segment
    (2, 6, 127, 64, 0, 64, 64, 64, 0, False, True),      # a second segment of one pixel
    (1, 10, 252, 32, 0, 32, 128, 128, 0, False, False),  # two whole segments, N = 128 (taps unstacked)
]


@pytest.mark.parametrize("case", CASES, ids=[f"cin{c[5]}-cout{c[6]}-{c[1]}x{c[2]}" for c in CASES])
def test_conv3_matches_torch(case):
    B, H, W, ldx, xoff, cin, cout, ldo, ooff, f32, relu = case
    dn = _dn()
    g = torch.Generator().manual_seed(cin * 1000 + cout)
    x = torch.zeros(B, H, W, ldx)
    x[..., xoff:xoff + cin] = torch.randn(B, H, W, cin, generator=g)
    kp = dn.kp_of(cin)
    w = torch.zeros(cout, kp)
    w[:, :9 * cin] = torch.randn(cout, 9 * cin, generator=g) * 0.2
    bias = torch.randn(cout, generator=g)
    xb, wb = x.to(torch.bfloat16), w.to(torch.bfloat16)
    w_t = wb.float()[:, :9 * cin].reshape(cout, 3, 3, cin).permute(0, 3, 1, 2).contiguous()
    x_t = xb.float()[..., xoff:xoff + cin].permute(0, 3, 1, 2).contiguous()
    ref = F.conv2d(x_t, w_t, bias, padding=1)
    if relu:
        ref = F.relu(ref)
    ref = ref.permute(0, 2, 3, 1)
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    wt = dn.conv3_weights(wb.cuda(), cout, cin)
    if f32:
        out = torch.full((B, H, W, ldo), -7.0, dtype=torch.float32, device="cuda")
    else:
        out = torch.full((B, ldo // 8, H, W, 8), -7.0, dtype=torch.bfloat16, device="cuda")
    dn.conv3(dn.to_planar(xb).cuda(), cin, wt, cout, bias.cuda(), out, xoff=xoff, ooff=ooff, relu=relu, err=err)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    if not f32:
        out = dn.from_planar(out)
    got = out[..., ooff:ooff + cout].float().cpu()
    scale = ref.abs().max().item()
    if f32:
        assert (got - ref).abs().max().item() <= 2e-3 * scale, (got - ref).abs().max().item()
    else:
        assert torch.allclose(got, ref, rtol=1.0 / 128, atol=2e-3 * scale), (got - ref).abs().max().item()
    rest = torch.cat([out[..., :ooff], out[..., ooff + cout:]], dim=-1).float()
    assert torch.all(rest == -7.0)  # nothing written outside the output slice


def test_conv3_repeated_calls_and_large_frame():
    """A 1280x720 frame (10 segments x 90 row blocks over the persistent CTAs) twice in a row."""
    dn = _dn()
    g = torch.Generator().manual_seed(5)
    B, H, W, cin, cout = 1, 720, 1280, 96, 32
    xb = (torch.randn(B, H, W, cin, generator=g) * 0.5).to(torch.bfloat16)
    w = torch.zeros(cout, dn.kp_of(cin))
    w[:, :9 * cin] = torch.randn(cout, 9 * cin, generator=g) * 0.1
    wb = w.to(torch.bfloat16)
    w_t = wb.float()[:, :9 * cin].reshape(cout, 3, 3, cin).permute(0, 3, 1, 2).contiguous().cuda()
    ref = F.conv2d(xb.float().permute(0, 3, 1, 2).cuda(), w_t, padding=1).permute(0, 2, 3, 1)
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    wt = dn.conv3_weights(wb.cuda(), cout, cin)
    for _ in range(2):
        out = torch.zeros(B, H, W, cout, device="cuda")
        dn.conv3(dn.to_planar(xb).cuda(), cin, wt, cout, None, out, err=err)
        torch.cuda.synchronize()
        assert int(err.item()) == 0
        assert (out - ref).abs().max().item() <= 2e-3 * ref.abs().max().item()


def test_unet_forward_matches_oracle():
    """The whole U-Net forward (conv3 layers, chunk-planar pooling and upsampling, residual) against
    the float64 oracle's forward on the same bf16 weights and input: the GPU keeps bf16 activations,
    so the residual agrees to within 3e-2 of its scale (relative L2)."""
    from oracle import denoise_ref as R
    dn = _dn()
    net = dn.Denoiser(seed=3)
    sd = net.state_dict()
    g = torch.Generator().manual_seed(5)
    sd["c6"]["w"][:, :9 * 32] = torch.randn(3, 9 * 32, generator=g) * 0.05
    for name in sd:
        sd[name]["b"] = torch.randn(sd[name]["b"].shape, generator=g) * 0.02
    net.load_state_dict(sd)
    B, H, W = 2, 24, 136
    x0 = torch.zeros(B, H, W, 8)
    x0[..., :6] = torch.rand(B, H, W, 6, generator=g)
    x0 = x0.to(torch.bfloat16)
    base = torch.rand(B, H, W, 3, generator=g)
    pred = net.forward(x0.cuda(), base.cuda()).cpu().numpy().astype(np.float64)
    params = {n: (q["wb"].float().cpu().numpy().astype(np.float64), q["b"].cpu().numpy().astype(np.float64))
              for n, q in net.p.items()}
    ref, _ = R.forward(params, x0.float().numpy().astype(np.float64), base.numpy().astype(np.float64))
    rb = base.numpy().astype(np.float64)
    assert np.linalg.norm((pred - rb) - (ref - rb)) <= 3e-2 * np.linalg.norm(ref - rb)
    assert net.error_word() == 0
