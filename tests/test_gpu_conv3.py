"""The TMA-staged 3x3 convolution (gpsb_dn_conv3, csrc/conv3x3.cu) against PyTorch's fp32
convolution of the same bf16-rounded operands, for every output width the kernel instantiates
(16 .. 192 channels), the input widths of the U-Net and of its data gradients (8 .. 192), images
whose width is not a multiple of the 128-pixel segment and whose height is not a multiple of the
row block, batches, channel slices of wider tensors (input offset, output offset), bf16 and fp32
outputs, bias and ReLU. Tolerance: fp32 accumulation order (2e-3 of the output's scale), or one
bf16 rounding for bf16 outputs. The whole U-Net on this engine is compared with the earlier
implicit-im2col engine."""
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
    (1, 9, 300, 40, 8, 24, 96, 96, 0, True, False),      # data gradient of c5a (96 out), offset input
    (1, 4, 129, 64, 0, 64, 192, 200, 8, True, False),    # data gradient of c4a (192 out), offset output
    (3, 8, 128, 8, 0, 8, 16, 16, 0, True, False),        # N = 16 with 16 outputs
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
    dt = torch.float32 if f32 else torch.bfloat16
    out = torch.full((B, H, W, ldo), -7.0, dtype=dt, device="cuda")
    dn.conv3(xb.cuda(), cin, wt, cout, bias.cuda(), out, xoff=xoff, ooff=ooff, relu=relu, err=err)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
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
        dn.conv3(xb.cuda(), cin, wt, cout, None, out, err=err)
        torch.cuda.synchronize()
        assert int(err.item()) == 0
        assert (out - ref).abs().max().item() <= 2e-3 * ref.abs().max().item()


def test_unet_engines_agree():
    """The whole U-Net forward on conv3 and on the implicit-im2col engine (both bf16 activations,
    fp32 accumulation): the predictions differ only by the rounding of the activations."""
    dn = _dn()
    a = dn.Denoiser(seed=3, engine="tma")
    b = dn.Denoiser(seed=3, engine="cp.async")
    g = torch.Generator().manual_seed(9)
    B, H, W = 2, 64, 200
    x = (torch.rand(B, H, W, 8, generator=g)).to(torch.bfloat16).cuda()
    base = torch.rand(B, H, W, 3, generator=g).cuda()
    pa = a.forward(x, base).clone()
    pb = b.forward(x, base).clone()
    torch.cuda.synchronize()
    ra, rb = pa - base, pb - base
    assert (ra - rb).abs().max().item() <= 2e-2 * rb.abs().max().item() + 1e-6
    assert a.error_word() == 0 and b.error_word() == 0
