"""CPU checks of the oracle's own tooling for the large parity cases:
* the threaded form of the O2 mirror (stages split over host threads, subpixel winners by a packed
  64-bit minimum) equals the literal sequential form (two passes over the recorded writes,
  shaders/gps_splat.wgsl:276-281) bit for bit, for every method and the primitive path;
* the oracle's PLY reader (oracle/ply.py, a restatement of crates/gps-io/src/lib.rs:260-373) gives
  the same 64-byte records and SH coefficients as the renderer's loader."""
import numpy as np
import pytest

import oracle as O
from conftest import load_package
from oracle import ply

PKG = load_package()
M, Cal, RP = PKG.Method, PKG.Calibration, PKG.RenderPath
W, H = 80, 48


@pytest.fixture(scope="module")
def scene():
    from gps_pbvr_web_b200 import scenes
    g, sh, deg, _ = ply.read_ply(scenes.cluster_scene(3000, seed=5, degree=3))
    return g, sh, deg


def cam(d):
    return PKG.OrbitCamera(target=(0.0, 0.0, 0.0), distance=d, yaw=0.6, pitch=0.25, up=(0.0, -1.0, 0.0),
                           fov_y=0.9).to_camera(W, H)


CASES = [
    ("GPS", dict(method=M.Gps)),
    ("GPS primitive", dict(method=M.Gps, path=RP.Primitive)),
    ("Proportional C0", dict(method=M.Proportional, pbvr=dict(calibration=Cal.None_))),
    ("Extinction C3+R", dict(method=M.Extinction, pbvr=dict(calibration=Cal.PerSplatFootprint,
                                                            radial_correction=True))),
    ("ViewConditioned", dict(method=M.ViewConditioned, pbvr=dict(calibration=Cal.None_, base_k=4096.0))),
    ("ScreenOccupancy", dict(method=M.ScreenOccupancy)),
]


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("side", [1, 2])
def test_threaded_o2_equals_sequential(scene, case, side):
    g, sh, deg = scene
    kw = dict(case[1])
    pb = kw.pop("pbvr", {})
    p = PKG.RenderParams(spp_side=side, max_points_per_splat=2048, **kw)
    for k, v in pb.items():
        setattr(p.pbvr, k, v)
    lut = O.radius_lut()
    for d in (3.0, 9.0):
        c = cam(d).to_array()
        a = O.o2_render_ensembles(g, sh, deg, lut, W, H, side, c, p.to_c(), 7, 2, want_counts=True, want_packed=True)
        b = O.o2_render_ensembles(g, sh, deg, lut, W, H, side, c, p.to_c(), 7, 2, want_counts=True, want_packed=True,
                                  threads=4)
        assert np.array_equal(a[0].view(np.uint32), b[0].view(np.uint32))
        assert np.array_equal(a[1], b[1]), (a[1].tolist(), b[1].tolist())
        assert np.array_equal(a[2], b[2])
        assert np.array_equal(a[3], b[3])
        assert a[1][10] > 0  # the case writes subpixels


def test_threaded_o2_overflow_skip(scene):
    """An ensemble whose particle total passes 2^32 - 1 is skipped in both forms (gps_splat.wgsl:635-663)."""
    g, sh, deg = scene
    # Proportional C0: every splat in front of the camera reaches the cap of 2^24 particles
    p = PKG.RenderParams(spp_side=1, max_points_per_splat=1 << 24, density_scale=1e9, method=M.Proportional)
    p.pbvr.calibration = Cal.None_
    lut = O.radius_lut()
    c = cam(3.0).to_array()
    a = O.o2_render_ensembles(g, None, 0, lut, W, H, 1, c, p.to_c(), 3, 1, want_packed=True)
    b = O.o2_render_ensembles(g, None, 0, lut, W, H, 1, c, p.to_c(), 3, 1, want_packed=True, threads=3)
    assert a[1][7] == 1 and np.array_equal(a[1], b[1])
    assert np.array_equal(a[0], b[0]) and np.all(a[0] == 0)


def test_oracle_ply_reader_equals_renderer_loader():
    from gps_pbvr_web_b200 import scenes
    for deg in (0, 1, 3):
        data = scenes.cluster_scene(5000, seed=deg, degree=deg)
        g, sh, d, sc = ply.read_ply(data)
        g2, sh2, d2 = PKG.load_ply(data)
        assert d == d2 == deg
        assert np.array_equal(g.view(np.uint32), g2.view(np.uint32))
        if deg:
            assert np.array_equal(sh.view(np.uint32), np.asarray(sh2, np.float32).reshape(sh.shape).view(np.uint32))
        assert np.array_equal(sc["opacity"], g[:, 3].astype(np.float64))
