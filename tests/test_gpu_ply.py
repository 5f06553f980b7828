"""GPU-side PLY decode (gpsb_load_ply_device) against the host loader (gpsb_load_ply, the gps-io
restatement): identical splats (opacity within one float ulp: the logistic's double exp may
differ in its last bit between the host's libm and the device) and SH, identical error messages
for a non-finite value, ASCII refused; the decoded scene renders like the host-loaded one."""
import numpy as np
import pytest

from conftest import load_package

pytestmark = pytest.mark.gpu
PKG = load_package()


def _compare(data):
    g_h, sh_h, d_h = PKG.load_ply(data)
    g_d, sh_d, d_d = PKG.load_ply_device(data)
    g_d = g_d.cpu().numpy()
    assert d_h == d_d and g_d.shape == g_h.shape
    mask = np.ones(16, bool)
    mask[3] = False
    assert np.array_equal(g_d[:, mask], g_h[:, mask])
    op_h, op_d = g_h[:, 3].view(np.int32), g_d[:, 3].view(np.int32)
    assert np.abs(op_h.astype(np.int64) - op_d).max() <= 1
    assert np.array_equal(sh_d.cpu().numpy(), np.asarray(sh_h).reshape(-1))
    return g_h, sh_h, d_h


def test_device_decode_matches_host():
    from gps_pbvr_web_b200 import scenes
    _compare(scenes.cluster_scene(50_000, seed=7, degree=3))
    _compare(scenes.cluster_scene(10_000, seed=8, degree=1))
    _compare(scenes.uniform_scene(20_000, seed=9))


def test_non_finite_and_ascii_errors():
    from gps_pbvr_web_b200 import scenes
    data = bytearray(scenes.uniform_scene(100, seed=1))
    head_end = data.index(b"end_header\n") + len(b"end_header\n")
    names = [l.split()[-1] for l in data[:head_end].decode().splitlines() if l.startswith("property")]
    stride = 4 * len(names)
    off = head_end + 17 * stride + 4 * names.index("scale_1")
    data[off:off + 4] = np.array([np.nan], "<f4").tobytes()
    with pytest.raises(PKG.GpsError) as eh:
        PKG.load_ply(bytes(data))
    with pytest.raises(PKG.GpsError) as ed:
        PKG.load_ply_device(bytes(data))
    assert ed.value.message == eh.value.message == "non-finite value in 'scale' at vertex 17"
    ascii_ply = b"ply\nformat ascii 1.0\nelement vertex 1\n" + b"".join(
        b"property float " + n.encode() + b"\n" for n in ["x", "y", "z", "f_dc_0", "f_dc_1", "f_dc_2", "opacity",
                                                          "scale_0", "scale_1", "scale_2", "rot_0", "rot_1", "rot_2",
                                                          "rot_3"]) + b"end_header\n" + b"0 " * 13 + b"1\n"
    PKG.load_ply(ascii_ply)
    with pytest.raises(PKG.GpsError):
        PKG.load_ply_device(ascii_ply)


def test_device_decoded_scene_renders_like_host_loaded():
    import torch
    from gps_pbvr_web_b200 import scenes
    data = scenes.cluster_scene(30_000, seed=3, degree=3)
    g_h, sh_h, d = PKG.load_ply(data)
    g_d, sh_d, _ = PKG.load_ply_device(data)
    W, H = 96, 64
    cam = PKG.OrbitCamera(target=(0.0, 0.0, 0.0), distance=6.0, yaw=0.3, pitch=0.2, up=(0.0, -1.0, 0.0),
                          fov_y=0.9).to_camera(W, H)
    p = PKG.RenderParams(spp_side=1, max_points_per_splat=4096, method=PKG.Method.Extinction)
    out = []
    for dev in (False, True):
        r = PKG.GpsRenderer(W, H, 1)
        if dev:
            r.set_gaussians_device(g_d.data_ptr(), g_d.shape[0], sh_d.data_ptr(), sh_d.numel(), d)
        else:
            r.set_gaussians_sh(g_h, sh_h, d)
        r.render_ensembles(cam, p, 5, 4)
        out.append(np.asarray(r.read_accum()))
        r.close()
    same_op = np.array_equal(g_h[:, 3], g_d.cpu().numpy()[:, 3])
    if same_op:
        assert np.array_equal(out[0], out[1])
    else:
        assert np.abs(out[0] - out[1]).max() < 0.5  # one-ulp opacities may move a few particles
