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
    dn.conv_dw(dn.to_planar(dyb).cuda(), dn.to_planar(xb), cin, cout, dw, err=err)  # chunk-planar operands
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


def _rand_frame(B, H, W, seed):
    import torch
    g = torch.Generator().manual_seed(seed)
    x0 = torch.zeros(B, H, W, 8)
    x0[..., :6] = torch.rand(B, H, W, 6, generator=g)
    base = torch.rand(B, H, W, 3, generator=g)
    target = (base + 0.1 * torch.randn(B, H, W, 3, generator=g)).clamp(0, 1)
    return x0.to(torch.bfloat16), base, target


def test_unet_gradients_match_oracle():
    """Every layer's weight and bias gradient of the GPU backward pass against the float64 oracle
    on the same bf16 weights and inputs (relative L2 error <= 5e-2: the GPU keeps bf16 activations)."""
    import torch
    from oracle import denoise_ref as R
    dn = _dn()
    net = dn.Denoiser(seed=3)
    sd = net.state_dict()
    g = torch.Generator().manual_seed(5)
    sd["c6"]["w"][:, :9 * 32] = torch.randn(3, 9 * 32, generator=g) * 0.05
    for name in sd:
        sd[name]["b"] = torch.randn(sd[name]["b"].shape, generator=g) * 0.02
    net.load_state_dict(sd)
    B, H, W = 2, 16, 16
    x0, base, target = _rand_frame(B, H, W, 1)
    net.zero_grad()
    net.forward(x0.cuda(), base.cuda())
    loss = net.backward(x0.cuda(), base.cuda(), target.cuda())
    torch.cuda.synchronize()
    params = {n: (q["wb"].float().cpu().numpy().astype(np.float64), q["b"].cpu().numpy().astype(np.float64))
              for n, q in net.p.items()}
    loss_ref, gref = R.loss_and_grads(params, x0.float().numpy().astype(np.float64), base.numpy().astype(np.float64),
                                      target.numpy().astype(np.float64))
    assert abs(loss.item() / (3 * B * H * W) - loss_ref) <= 1e-2 * loss_ref
    for name, q in net.p.items():
        cin = q["cin"]
        gw = q["gw"].cpu().numpy()[:, :9 * cin]
        rw = gref[name][0]
        assert np.linalg.norm(gw - rw) <= 5e-2 * np.linalg.norm(rw) + 1e-9, (name, np.linalg.norm(gw - rw) / np.linalg.norm(rw))
        gb, rb = q["gb"].cpu().numpy(), gref[name][1]
        assert np.linalg.norm(gb - rb) <= 5e-2 * np.linalg.norm(rb) + 1e-9, name
    assert net.error_word() == 0


def test_adam_update_matches_formula():
    import ctypes as C
    import torch
    dn = _dn()
    n = 1000
    g = torch.Generator().manual_seed(2)
    w0, gr = torch.randn(n, generator=g), torch.randn(n, generator=g)
    w, m, v = w0.clone().cuda(), torch.zeros(n, device="cuda"), torch.zeros(n, device="cuda")
    wb = torch.zeros(n, dtype=torch.bfloat16, device="cuda")
    L = PKG.abi.lib()
    for t in (1, 2):
        assert L.gpsb_dn_adam(C.c_void_p(w.data_ptr()), C.c_void_p(gr.cuda().data_ptr()), C.c_void_p(m.data_ptr()),
                              C.c_void_p(v.data_ptr()), n, 1e-3, 0.9, 0.999, 1e-8, t, C.c_void_p(wb.data_ptr()),
                              dn._stream()) == 0
    torch.cuda.synchronize()
    rm, rv, rw = np.zeros(n), np.zeros(n), w0.numpy().astype(np.float64)
    for t in (1, 2):
        rm = 0.9 * rm + 0.1 * gr.numpy()
        rv = 0.999 * rv + 0.001 * gr.numpy() ** 2
        rw = rw - 1e-3 * (rm / (1 - 0.9 ** t)) / (np.sqrt(rv / (1 - 0.999 ** t)) + 1e-8)
    assert np.abs(w.cpu().numpy() - rw).max() < 1e-6
    assert torch.equal(wb.cpu(), w.cpu().to(torch.bfloat16))


def test_training_reduces_loss():
    """Sixty Adam steps (lr 2e-3) on one fixed batch whose target is a function of the input
    features lower its L1 loss as the float64 oracle's own Adam run does (0.155 -> 0.118 from the
    same initialisation scheme): below 0.85 of the first step's loss."""
    import torch
    dn = _dn()
    net = dn.Denoiser(seed=0)
    x0, base, _ = _rand_frame(4, 32, 32, 9)
    target = 0.5 * base + 0.4 * x0[..., 3:4].float()
    x0, base, target = x0.cuda(), base.cuda(), target.cuda()
    losses = [net.train_step(x0, base, target, lr=2e-3).item() for _ in range(60)]
    assert losses[-1] < 0.85 * losses[0], losses
    assert sum(losses[-10:]) < sum(losses[:10]), losses
    assert net.error_word() == 0


def test_feature_accumulation():
    """Denoiser features of the renderer: after one ensemble the squared-colour sums equal the
    accumulated colour squared (bit for bit), alpha lies in [0, 1] with a depth only where covered;
    after four the sums of squares bound the squared sums (Cauchy-Schwarz)."""
    import torch
    from gps_pbvr_web_b200 import scenes
    W, H = 160, 96
    splats, sh, deg = PKG.load_ply(scenes.cluster_scene(20_000, seed=4, degree=1))
    r = PKG.GpsRenderer(W, H, 2)
    r.set_gaussians_sh(splats, sh, deg)
    cam = PKG.OrbitCamera(target=(0.0, 0.0, 0.0), distance=7.0, yaw=0.3, pitch=0.2, up=(0.0, -1.0, 0.0),
                          fov_y=0.9).to_camera(W, H)
    p = PKG.RenderParams(spp_side=2, max_points_per_splat=4096, method=PKG.Method.Extinction)
    feat = torch.zeros(W * H * 8, device="cuda")
    r.set_feature_accum(feat)
    r.render_ensembles(cam, p, 10, 1)
    acc = torch.from_numpy(np.asarray(r.read_accum(), dtype=np.float32).reshape(-1, 4))
    f = feat.reshape(-1, 8).cpu()
    assert torch.equal(f[:, :3], acc[:, :3] * acc[:, :3])
    assert float(f[:, 3].min()) >= 0.0 and float(f[:, 3].max()) <= 1.0
    assert torch.all((f[:, 4] > 0) == (f[:, 3] > 0))
    assert float(f[:, 3].max()) > 0.5
    r.render_ensembles(cam, p, 11, 3)
    acc = torch.from_numpy(np.asarray(r.read_accum(), dtype=np.float32).reshape(-1, 4)).double()
    f = feat.reshape(-1, 8).cpu().double()
    assert torch.all(f[:, :3] * 4 >= acc[:, :3] ** 2 * (1 - 1e-5))
    assert torch.all(f[:, 5:] == 0)
    r.set_feature_accum(None)
    r.close()


def test_trained_network_gain():
    """What the trained network (committed weights) gains over the method without it on a held-out
    scene and camera: the denoised 4-ensemble frame against a 64-ensemble reference (disjoint seeds)
    beats the plain 4-ensemble frame by more than 6 dB and the plain 16-ensemble frame outright; the
    variance check passes, so the denoiser is used."""
    import torch
    from gps_pbvr_web_b200 import scenes
    from gps_pbvr_web_b200 import denoise_train as T
    dn = _dn()
    net = dn.Denoiser()
    gate = dn.load_weights(net)
    W, H = 640, 360
    splats, sh, deg = PKG.load_ply(scenes.cluster_scene(150_000, seed=31, degree=3))
    r = PKG.GpsRenderer(W, H, 1)
    r.set_gaussians_sh(splats, sh, deg)
    cam = PKG.OrbitCamera(target=(0.0, 0.0, 0.0), distance=6.0, yaw=1.1, pitch=0.3, up=(0.0, -1.0, 0.0),
                          fov_y=0.9).to_camera(W, H)
    p = T.params(PKG)
    r.render_ensembles(cam, p, 900_000, 64)
    ref = T.mean_rgb(torch.from_numpy(r.read_accum()).cuda())
    out, used, check = dn.render_denoised(r, net, cam, p, 5, gate_limit=gate)
    assert used and check <= gate
    plain = {}
    for n in (4, 16):
        r.reset_accum()
        r.render_ensembles(cam, p, 5, n)
        plain[n] = T.psnr(T.mean_rgb(torch.from_numpy(r.read_accum()).cuda()), ref)[0]
    got = T.psnr(out, ref)[0]
    assert got > plain[4] + 6.0 and got > plain[16], (got, plain)
    assert net.error_word() == 0
    r.close()
