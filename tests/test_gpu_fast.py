"""PBVR fast decisions (pbvr_fast in csrc/kernels.cu): the approximation constants hold over every
input they can get (exhaustive check on the device), the fast answers never disagree with the exact
path (validation mode runs both for every particle and counts disagreements), and turning the fast
decisions on leaves every output bit-identical: accumulated image, points and subpixel writes."""
import numpy as np
import pytest

from _parity import PKG

pytestmark = pytest.mark.gpu

M, Cal = PKG.Method, PKG.Calibration
W, H, N = 640, 360, 150_000
VIEWS = (("near", 2.5), ("mid", 7.0), ("far", 20.0))

CASES = [
    # name, method, calibration, radial, centre depth, jitter
    ("Extinction C3+R", M.Extinction, Cal.PerSplatFootprint, True, False, True),
    ("Extinction C3+R centre-depth", M.Extinction, Cal.PerSplatFootprint, True, True, True),
    ("Extinction C3 no-jitter", M.Extinction, Cal.PerSplatFootprint, False, False, False),
    ("Proportional C0", M.Proportional, Cal.None_, False, False, True),
    ("ViewConditioned C0", M.ViewConditioned, Cal.None_, False, False, True),
]


@pytest.fixture(scope="module")
def scene():
    from gps_pbvr_web_b200 import scenes
    return PKG.load_ply(scenes.cluster_scene(N, seed=0, degree=3))


def cams():
    return [(n, PKG.OrbitCamera(target=(0.0, 0.0, 0.0), distance=d, yaw=0.6, pitch=0.25, up=(0.0, -1.0, 0.0),
                                fov_y=0.9).to_camera(W, H)) for n, d in VIEWS]


def params(case):
    _, method, cal, radial, centre, jitter = case
    p = PKG.RenderParams(spp_side=1, max_points_per_splat=16384, method=method)
    p.pbvr.calibration = cal
    p.pbvr.radial_correction = radial
    p.pbvr.centre_depth = centre
    p.pbvr.low_pass_jitter = jitter
    if method == M.ViewConditioned:
        p.pbvr.base_k = 4096.0
    return p


def render(r, cam, p, mode, ens=3, seed=11):
    r.set_fast_decisions(mode)
    r.reset_accum()
    r.reset_stats()
    r.render_ensembles(cam, p, seed, ens)
    st = r.read_stats()
    return r.read_accum(), st, r.debug_fast_counts()


def test_fast_bounds_hold():
    r = PKG.GpsRenderer(16, 16, 1)
    ratios = r.debug_fast_bounds()
    r.close()
    print("error / bound: log(u) %.3f log(v) %.3f sincos %.3f radius %.3f max radius %.3f exp %.3f" % tuple(ratios))
    assert np.all(np.isfinite(ratios)) and np.all(ratios > 0.0) and np.all(ratios <= 1.0), ratios


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_fast_decisions_agree_with_exact_path(scene, case):
    splats, sh, deg = scene
    r = PKG.GpsRenderer(W, H, 1)
    r.set_gaussians_sh(splats, sh, deg)
    p = params(case)
    for name, cam in cams():
        a0, s0, _ = render(r, cam, p, 0)
        a2, s2, (undecided2, mismatch) = render(r, cam, p, 2)
        a1, s1, (undecided1, _) = render(r, cam, p, 1)
        print(f"{case[0]} {name}: particles {s0.particles} points {s0.points} writes {s0.subpixel_writes} "
              f"undecided {undecided2} ({undecided2 / max(s0.particles, 1):.4f})")
        assert mismatch == 0, (name, mismatch)
        assert s0.particles >= s0.points >= s0.subpixel_writes and undecided2 <= s0.particles
        for a, s in ((a1, s1), (a2, s2)):
            assert np.array_equal(a.view(np.uint32), a0.view(np.uint32)), name
            assert s.counters() == s0.counters() and s.subpixel_writes == s0.subpixel_writes, name
            assert s.particles == s0.particles, name
        assert undecided1 <= undecided2
    assert r.debug_error_word() == 0
    r.close()


def test_fast_decisions_near_view_mostly_decided(scene):
    splats, sh, deg = scene
    r = PKG.GpsRenderer(W, H, 1)
    r.set_gaussians_sh(splats, sh, deg)
    _, cam = cams()[0]
    _, st, (undecided, mismatch) = render(r, cam, params(CASES[0]), 2)
    r.close()
    # the near view writes few of its particles: the fast decisions settle most of the rest
    assert mismatch == 0 and st.points > 0 and st.subpixel_writes < 0.05 * st.particles
    assert undecided < 0.4 * st.particles, (undecided, st.particles, st.subpixel_writes)


def test_fast_decisions_bench_scene_validated():
    """The 560k-Gaussian benchmark scene at 1280x720 (near / mid / far orbit views, 2 ensembles each):
    every particle's fast answer agrees with the exact path, and the images match bit for bit."""
    from gps_pbvr_web_b200 import scenes
    splats, sh, deg = PKG.load_ply(scenes.cluster_scene(560_000, seed=0, degree=3))
    w, h = 1280, 720
    r = PKG.GpsRenderer(w, h, 1)
    r.set_gaussians_sh(splats, sh, deg)
    p = params(CASES[0])
    total = 0
    for d in (2.5, 7.0, 20.0):
        cam = PKG.OrbitCamera(target=(0.0, 0.0, 0.0), distance=d, yaw=0.6, pitch=0.25, up=(0.0, -1.0, 0.0),
                              fov_y=0.9).to_camera(w, h)
        a2, s2, (_, mismatch) = render(r, cam, p, 2, ens=2, seed=3)
        a1, s1, _ = render(r, cam, p, 1, ens=2, seed=3)
        assert mismatch == 0, (d, mismatch)
        assert np.array_equal(a1.view(np.uint32), a2.view(np.uint32)) and s1.counters() == s2.counters()
        total += s2.particles
    assert total > 3e9 and r.debug_error_word() == 0
    r.close()


def test_scene_reloads_reuse_buffers_and_match_fresh_renderers():
    """Reloading scenes of different sizes into one renderer (the spare scene buffers swap, the
    per-ensemble buffers grow) renders exactly what a fresh renderer renders."""
    from gps_pbvr_web_b200 import scenes
    small = PKG.load_ply(scenes.cluster_scene(20_000, seed=5, degree=1))
    large = PKG.load_ply(scenes.cluster_scene(120_000, seed=6, degree=3))
    _, cam = cams()[1]
    p = params(CASES[0])

    def fresh(sc):
        r = PKG.GpsRenderer(W, H, 1)
        r.set_gaussians_sh(*sc)
        out = render(r, cam, p, 1, ens=2, seed=9)[0]
        r.close()
        return out

    want_small, want_large = fresh(small), fresh(large)
    r = PKG.GpsRenderer(W, H, 1)
    for sc, want in ((small, want_small), (large, want_large), (small, want_small), (large, want_large)):
        r.set_gaussians_sh(*sc)
        got = render(r, cam, p, 1, ens=2, seed=9)[0]
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    assert r.debug_error_word() == 0
    r.close()
