"""The frame-loop session on the real renderer: Auto path on a GPS scene converges to the target
through the probe and the chosen path; PBVR through particles with adaptive LOD; and the
half-resolution mode (render at ceil(w/2) x ceil(h/2), composite at w x h, lib.rs:333-353)."""
import importlib

import numpy as np
import pytest

from conftest import load_package

pytestmark = pytest.mark.gpu
PKG = load_package()
S = importlib.import_module(PKG.__name__ + ".session")


def _scene(r):
    from gps_pbvr_web_b200 import scenes
    splats, sh, deg = PKG.load_ply(scenes.cluster_scene(30_000, seed=2, degree=1))
    r.set_gaussians_sh(splats, sh, deg)


def test_session_auto_path_reaches_target():
    W, H = 128, 96
    r = PKG.GpsRenderer(W, H, 1)
    _scene(r)
    cam = PKG.OrbitCamera(target=(0.0, 0.0, 0.0), distance=4.0, yaw=0.4, pitch=0.2, up=(0.0, -1.0, 0.0),
                          fov_y=0.9).to_camera(W, H)
    s = S.FrameSession(renderer=r)
    s.configure(PKG.RenderParams(spp_side=1, max_points_per_splat=4096), per_frame=4, target=16)
    s.set_render_path(2, 0.1)  # a tiny threshold: the probe picks the sorted path
    s.set_camera(cam)
    t = 0.0
    for _ in range(40):
        t += 16.7
        s.frame(t)
        if r.accumulated() >= 16:
            break
    r.wait_idle()
    assert r.accumulated() >= 16
    assert s.state()["sorted_active"] == 1 and s.state()["last_demand"] > 0
    s.close()
    r.close()


def test_session_pbvr_adaptive_lod():
    W, H = 128, 96
    r = PKG.GpsRenderer(W, H, 1)
    _scene(r)
    cam = PKG.OrbitCamera(target=(0.0, 0.0, 0.0), distance=6.0, yaw=0.4, pitch=0.2, up=(0.0, -1.0, 0.0),
                          fov_y=0.9).to_camera(W, H)
    p = PKG.RenderParams(spp_side=1, max_points_per_splat=4096, method=PKG.Method.Extinction)
    s = S.FrameSession(renderer=r)
    s.configure(p, per_frame=1, target=12)
    s.set_lod(True, 33.3, 256)
    s.set_camera(cam)
    t = 0.0
    for _ in range(60):
        t += 5.0
        s.frame(t)
    r.wait_idle()
    assert r.accumulated() == 12 and s.state()["sorted_active"] == 0
    s.close()
    r.close()


def test_half_resolution_mode():
    W, H = 161, 97
    r = PKG.GpsRenderer(W, H, 1)
    _scene(r)
    w2, h2 = (W + 1) // 2, (H + 1) // 2
    r.resize(w2, h2, 1)
    cam = PKG.OrbitCamera(target=(0.0, 0.0, 0.0), distance=6.0, yaw=0.4, pitch=0.2, up=(0.0, -1.0, 0.0),
                          fov_y=0.9).to_camera(w2, h2)
    p = PKG.RenderParams(spp_side=1, max_points_per_splat=4096)
    r.render_ensembles(cam, p, 1, 4)
    img = np.asarray(r.composite(p, W, H))
    assert img.size == W * H * 4
    small = np.asarray(r.composite(p, w2, h2))
    assert small.size == w2 * h2 * 4
    # the upsampling composite (gps_composite.wgsl:41-55) of the half-size accumulation at the odd
    # output size, and the plain one at its own size, equal the O2 mirror byte for byte
    import oracle as O
    acc = r.read_accum()
    for ow, oh, got in ((W, H, img), (w2, h2, small)):
        want = O.o2_composite(acc, w2, h2, p.exposure, p.srgb_output, ow, oh)
        assert np.array_equal(np.asarray(got).reshape(-1, 4), want), (ow, oh)
    r.close()


def test_trajectory_graph_matches_the_direct_path():
    """The captured trajectory (16 orbit cameras x 3 ensembles) equals the directly encoded one
    bit for bit, on the capture and on a replay; new seeds re-capture and still match."""
    import torch
    W, H = 96, 64
    r = PKG.GpsRenderer(W, H, 1)
    _scene(r)
    st = torch.cuda.Stream()
    r.set_stream(st.cuda_stream)
    cams = [PKG.OrbitCamera(target=(0.0, 0.0, 0.0), distance=5.0, yaw=0.4 * k, pitch=0.2, up=(0.0, -1.0, 0.0),
                            fov_y=0.9).to_camera(W, H) for k in range(16)]
    p = PKG.RenderParams(spp_side=1, max_points_per_splat=4096, method=PKG.Method.Extinction)
    a = torch.zeros(16 * W * H * 4, device="cuda")
    b = torch.zeros_like(a)
    r.render_trajectory(cams, p, 11, 3, a.data_ptr())
    r.wait_idle()
    for _ in range(2):
        b.fill_(-1.0)
        r.render_trajectory_graph(cams, p, 11, 3, b.data_ptr())
        r.wait_idle()
        assert torch.equal(a, b)
    r.render_trajectory(cams, p, 40, 3, a.data_ptr())
    r.render_trajectory_graph(cams, p, 40, 3, b.data_ptr())
    r.wait_idle()
    assert torch.equal(a, b) and r.debug_error_word() == 0
    r.close()


def test_autotuner_sweeps_and_shapes_do_not_change_results():
    """The autotuner times every particle launch shape through the captured graph and returns the
    fastest; every shape renders the same accumulation bit for bit."""
    import torch
    from gps_pbvr_web_b200 import autotune
    W, H = 96, 64
    r = PKG.GpsRenderer(W, H, 1)
    _scene(r)
    st = torch.cuda.Stream()
    with torch.cuda.stream(st):
        cams = [PKG.OrbitCamera(target=(0.0, 0.0, 0.0), distance=5.0, yaw=0.5 * k, pitch=0.2, up=(0.0, -1.0, 0.0),
                                fov_y=0.9).to_camera(W, H) for k in range(2)]
        p = PKG.RenderParams(spp_side=1, max_points_per_splat=4096, method=PKG.Method.Extinction)
        best, results = autotune.tune(r, cams, p, ensembles=2, reps=2)
        assert len(results) == len(autotune.PARTICLE_SPACE) and best in autotune.PARTICLE_SPACE
        assert all(ms > 0 for _, ms in results)
        outs = []
        for shape in (autotune.PARTICLE_SPACE[0], autotune.PARTICLE_SPACE[-1], best):
            r.set_tuning(**shape)
            o = torch.zeros(2 * W * H * 4, device="cuda")
            r.render_trajectory(cams, p, 3, 2, o.data_ptr())
            r.wait_idle()
            outs.append(o)
        assert torch.equal(outs[0], outs[1]) and torch.equal(outs[0], outs[2])
    r.close()
