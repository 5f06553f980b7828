"""The error propagation of the renderer's PBVR fast decisions, checked on the CPU: the oracle
restates the decisions with every hardware approximation replaced by the exact value pushed to the
edge of its assumed error bound (random signs, all +, all -), and whenever that restated fast path
answers "not a point" or "a point off screen" the exact path must agree, over every particle of
a frame. (The device's own approximations are checked against those bounds exhaustively on the
GPU, tests/test_gpu_fast.py.)"""
import pytest

import oracle as O
from conftest import load_package

PKG = load_package()


@pytest.fixture(scope="module")
def scene():
    from gps_pbvr_web_b200 import scenes
    return PKG.load_ply(scenes.cluster_scene(6000, seed=4, degree=1))


def _params(method, cal, radial=True, jitter=True, centre=False):
    p = PKG.RenderParams(spp_side=1, max_points_per_splat=256, method=method)
    p.pbvr.calibration = cal
    p.pbvr.radial_correction = radial
    p.pbvr.low_pass_jitter = jitter
    p.pbvr.centre_depth = centre
    if method == PKG.Method.ViewConditioned:
        p.pbvr.base_k = 256.0
    return p


CASES = [
    ("Extinction C3+R", PKG.Method.Extinction, PKG.Calibration.PerSplatFootprint, True, True),
    ("Extinction C3 no-jitter", PKG.Method.Extinction, PKG.Calibration.PerSplatFootprint, False, False),
    ("Extinction C1+R", PKG.Method.Extinction, PKG.Calibration.ObjectZoom, True, True),
    ("Proportional C2+R", PKG.Method.Proportional, PKG.Calibration.PerSplatDepth, True, True),
    ("ViewConditioned C0 +R", PKG.Method.ViewConditioned, PKG.Calibration.None_, True, True),
]


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("mode,seed", [(0, 1), (0, 2), (1, 0), (2, 0)])
def test_fast_decisions_hold_at_the_edge_of_their_bounds(scene, case, mode, seed):
    splats, sh, deg = scene
    w, h = 320, 180
    _, method, cal, radial, jitter = case
    p = _params(method, cal, radial, jitter)
    decided_total = particles_total = 0
    for d in (1.5, 2.5, 7.0):
        cam = PKG.OrbitCamera(target=(0.0, 0.0, 0.0), distance=d, yaw=0.6, pitch=0.25, up=(0.0, -1.0, 0.0),
                              fov_y=0.9).to_camera(w, h)
        particles, decided, wrong, points = O.o2_fast_check(splats, sh, deg, O_lut(), w, h, 1, cam.to_array(),
                                                            p.to_c(), 5, 1, perturb_seed=seed, mode=mode)
        assert wrong == 0, (d, wrong, decided, particles)
        assert particles > 0 and points <= particles
        decided_total += decided
        particles_total += particles
    assert decided_total > 0.3 * particles_total, (decided_total, particles_total)


def O_lut():
    from _parity import lut
    return lut()
