"""Bit-exact parity on the benchmarked workload itself: 560,000 clustered Gaussians with SH degree 3,
PBVR Extinction C3+R, spp 1, per-splat cap 16,384, 1280x720, the near / mid / far orbit views of the
benchmark, fast decisions on (the renderer's default). The CUDA renderer, called through the C ABI,
is compared with the O2 mirror oracle (threaded form) on per-splat counts, every packed subpixel
word (depth key << 32 | winner), every statistics counter and every accumulation word. The
reference path matched is render_ensembles (crates/gps-render/src/gps.rs:861-925) with prepare and
particle_pass (shaders/gps_splat.wgsl:617-720).

Cases: the far view with 2 ensembles; the mid view with 1 ensemble; the near view on a uniform
1/16 subset of the splats; one 64-ensemble batch at the far view (batch offsets of the persistent
particle kernel, per-ensemble list windows, ensemble-ordered accumulation); and a frame whose
particle total lies between 2^31 and 2^32 - 1 (particle offsets above the signed 32-bit range)."""
import os

import numpy as np
import pytest

import oracle as O
from _parity import PKG, stats_tuple
from oracle import ply

pytestmark = pytest.mark.gpu

W, H, CAP = 1280, 720, 16384
THREADS = os.cpu_count() or 1
VIEWS = {"near": 2.5, "mid": 7.0, "far": 20.0}


@pytest.fixture(scope="module")
def scene():
    from gps_pbvr_web_b200 import scenes
    g, sh, deg, _ = ply.read_ply(scenes.cluster_scene(560_000, seed=0, degree=3))
    return g, sh, deg


def camera(view, w=W, h=H):
    return PKG.OrbitCamera(target=(0.0, 0.0, 0.0), distance=VIEWS[view], yaw=0.6, pitch=0.25, up=(0.0, -1.0, 0.0),
                           fov_y=0.9).to_camera(w, h)


def c3r(cap=CAP, density=1.0):
    p = PKG.RenderParams(spp_side=1, max_points_per_splat=cap, method=PKG.Method.Extinction, density_scale=density)
    p.pbvr.calibration = PKG.Calibration.PerSplatFootprint
    p.pbvr.radial_correction = True
    return p


def compare(g, sh, deg, cam, p, first_seed, count, w=W, h=H):
    """Render on the GPU and in O2; assert every output equal; return the statistics tuple and the
    particle total (after the cap) of each ensemble."""
    r = PKG.GpsRenderer(w, h, 1)
    try:
        r.set_gaussians_sh(g, sh, deg)
        r.render_ensembles(cam, p, first_seed, count)
        acc = r.read_accum()
        st = stats_tuple(r.read_stats())
        oacc, ost, ocounts, opacked = O.o2_render_ensembles(g, sh, deg, O.radius_lut(), w, h, 1, cam.to_array(),
                                                            p.to_c(), first_seed, count, want_counts=True,
                                                            want_packed=True, threads=THREADS)
        assert st == tuple(int(x) for x in ost), (st, ost.tolist())
        for e in range(count):
            if ost[7] == 0:  # no ensemble skipped: every slot holds a compact list
                c = r.debug_counts(e)
                bad = np.flatnonzero(c != ocounts[e])
                assert bad.size == 0, f"ensemble {e}: {bad.size} per-splat counts differ, first {bad[:5].tolist()}"
            pk = r.debug_subpixels(e)
            bad = np.flatnonzero(pk != opacked[e])
            assert bad.size == 0, f"ensemble {e}: {bad.size} subpixel words differ, first {bad[:5].tolist()}: " \
                f"{[hex(int(pk[j])) for j in bad[:3]]} vs {[hex(int(opacked[e][j])) for j in bad[:3]]}"
        eq = acc.view(np.uint32) == oacc.view(np.uint32)
        assert eq.all(), f"{(~eq).sum()} accumulation words differ; max abs {np.abs(acc - oacc).max()}"
        return st, ocounts.sum(axis=1, dtype=np.uint64)
    finally:
        r.close()


def test_far_two_ensembles(scene):
    st, _ = compare(*scene, camera("far"), c3r(), 1, 2)
    assert st[10] > 1_000_000  # subpixel writes: the case is not empty


def test_mid_one_ensemble(scene):
    st, _ = compare(*scene, camera("mid"), c3r(), 5, 1)
    assert st[5] > 100_000_000  # candidates


def test_near_uniform_sixteenth(scene):
    g, sh, deg = scene
    st, _ = compare(g[::16].copy(), sh[::16].copy(), deg, camera("near"), c3r(), 9, 1)
    assert st[10] > 100_000


def test_far_64_ensemble_batch(scene):
    st, _ = compare(*scene, camera("far"), c3r(), 100, 64)
    assert st[8] == 64 and st[7] == 0


def test_particle_offsets_beyond_2_31(scene):
    """136 splats in front of the mid camera, each at the cap of 2^24 particles: 2,281,701,376
    particles in one ensemble, between 2^31 and 2^32 - 1 (the ensemble is not skipped)."""
    g, sh, deg = scene
    cam = camera("mid", 320, 180)
    R = np.asarray(cam.view_rot, np.float64).reshape(3, 3)
    z = (g[:, 0:3].astype(np.float64) - np.asarray(cam.view_pos, np.float64)) @ R[2]
    pick = np.flatnonzero((z > 1.0) & (g[:, 3] > 0.3))[:136]
    assert pick.size == 136
    p = c3r(cap=1 << 24, density=1e9)
    st, total = compare(g[pick].copy(), sh[pick].copy(), deg, cam, p, 3, 1, 320, 180)
    assert (1 << 31) < int(total[0]) < (1 << 32) and st[7] == 0, (int(total[0]), st)
