"""The denoised frame through the C ABI (gpsb_denoiser_*, gpsb_render_denoised: the network
sequenced by the library's C++ host code over the conv3 kernels, with host output buffers), against
the Python sequencing of the same kernels (denoise.Denoiser / denoise.render_denoised), and the
variance-check fallback to the plain accumulation."""
import numpy as np
import pytest

from conftest import load_package

pytestmark = pytest.mark.gpu
PKG = load_package()
torch = pytest.importorskip("torch")

W, H = 256, 192


def _dn():
    import importlib
    return importlib.import_module(PKG.__name__ + ".denoise")


@pytest.fixture(scope="module")
def setup():
    from gps_pbvr_web_b200 import scenes
    g, sh, deg = PKG.load_ply(scenes.cluster_scene(60_000, seed=4, degree=3))
    r = PKG.GpsRenderer(W, H, 1)
    r.set_gaussians_sh(g, sh, deg)
    cam = PKG.OrbitCamera(target=(0.0, 0.0, 0.0), distance=7.0, yaw=0.6, pitch=0.25, up=(0.0, -1.0, 0.0),
                          fov_y=0.9).to_camera(W, H)
    p = PKG.RenderParams(spp_side=1, max_points_per_splat=16384, method=PKG.Method.Extinction)
    p.pbvr.calibration = PKG.Calibration.PerSplatFootprint
    p.pbvr.radial_correction = True
    yield r, cam, p
    r.close()


def test_native_forward_equals_python_sequencing():
    dn = _dn()
    net = dn.Denoiser()
    dn.load_weights(net)
    nat = dn.NativeDenoiser()
    g = torch.Generator().manual_seed(2)
    x = torch.rand(1, 64, 136, 8, generator=g).to(torch.bfloat16).cuda()
    base = torch.rand(1, 64, 136, 3, generator=g).cuda()
    a = net.forward(x, base).clone()
    b = torch.zeros_like(a)
    nat.forward(x, base, b)
    torch.cuda.synchronize()
    assert torch.equal(a, b), (a - b).abs().max().item()
    nat.close()


def test_native_forward_graph_replay():
    """The first forward of a frame size launches the layers directly and captures them; later
    forwards replay the capture (gpsb_denoiser_graph_state). Every call, on new inputs and across a
    change of frame size and back, equals the Python sequencing bit for bit."""
    dn = _dn()
    net = dn.Denoiser()
    dn.load_weights(net)
    nat = dn.NativeDenoiser()
    g = torch.Generator().manual_seed(7)
    for H_, W_ in ((64, 136), (64, 136), (64, 136), (48, 96), (64, 136)):
        x = torch.rand(1, H_, W_, 8, generator=g).to(torch.bfloat16).cuda()
        base = torch.rand(1, H_, W_, 3, generator=g).cuda()
        a = net.forward(x, base).clone()
        b = torch.full_like(a, -1.0)
        nat.forward(x, base, b)
        torch.cuda.synchronize()
        assert torch.equal(a, b), (H_, W_, (a - b).abs().max().item())
        assert nat.graph_state() == 1  # this size's layers are captured (and replayed from now on)
    nat.close()


def test_render_denoised_through_the_c_abi(setup):
    r, cam, p = setup
    dn = _dn()
    net = dn.Denoiser()
    gate = dn.load_weights(net)
    rgb_py, used_py, chk_py = dn.render_denoised(r, net, cam, p, 1000, ensembles=4, gate_limit=gate)
    nat = dn.NativeDenoiser()
    rgb, used, chk = nat.render(r, cam, p, 1000, ensembles=4)
    assert used and used_py
    assert abs(chk - chk_py) <= 1e-4 * max(chk_py, 1e-6)
    assert np.array_equal(rgb, rgb_py.cpu().numpy())
    nat.close()


def test_render_denoised_falls_back_when_the_check_fails(setup):
    """With a limit below the frame's check value the plain accumulation of the fallback ensembles
    (the 4 rendered ones plus the next seeds) is returned, in the Python and the C sequencing."""
    r, cam, p = setup
    dn = _dn()
    net = dn.Denoiser()
    dn.load_weights(net)
    nat = dn.NativeDenoiser()
    rgb, used, chk = nat.render(r, cam, p, 2000, ensembles=4, gate_limit=1e-9, fallback_ensembles=16)
    assert not used and chk > 1e-9
    rgb_py, used_py, _ = dn.render_denoised(r, net, cam, p, 2000, ensembles=4, gate_limit=1e-9, fallback_ensembles=16)
    assert not used_py
    r.reset_accum()
    r.render_ensembles(cam, p, 2000, 16)
    acc = r.read_accum()
    plain = acc[:, :3] / np.maximum(acc[:, 3:4], 1.0)
    assert np.array_equal(rgb, plain.astype(np.float32))
    assert np.allclose(rgb_py.cpu().numpy(), plain, rtol=0, atol=1e-6)
    nat.close()
