"""Checks of the device maths that do not go through the O2 mirror (which shares csrc/fmath.h with
the kernels, so a mistake common to both would pass every bit-exact test):

* the per-particle stream seeds the particle kernel derives on the GPU (owner splat from the compact
  list, index k, particle_seed(i, k + 1, seed)) equal O1's restatement of gps-core's particle_seed
  (crates/gps-core/src/lib.rs:450-465) for every particle of several splats, including particles
  whose ensemble offset lies above 2^31;
* exp / log / sin / cos evaluated on the device, in the shared-memory-table form of the particle
  kernel and the global-table form of the other kernels, against libm in double precision over the
  inputs the kernels see: every Box-Muller uniform, every angle 2 pi U, and wide sweeps."""
import numpy as np
import pytest

import oracle as O
from _parity import PKG

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

M, Cal = PKG.Method, PKG.Calibration


def o1_seeds(i, k0, k1, seed):
    return np.array([O.particle_seed(True, int(i), k + 1, seed) for k in range(k0, k1)], np.uint32)


def check_splat(r, counts, i, seed, offsets, limit=4096):
    """Every particle of splat i (at most `limit` from each end) against O1."""
    n = int(counts[i])
    spans = [(0, n)] if n <= 2 * limit else [(0, limit), (n - limit, n)]
    for k0, k1 in spans:
        got = r.debug_particle_seeds(0, int(offsets[i]) + k0, k1 - k0)
        assert np.all(got[:, 0] == i), (i, np.unique(got[:, 0])[:5])
        assert np.array_equal(got[:, 1], np.arange(k0, k1, dtype=np.uint32))
        want = o1_seeds(i, k0, k1, seed)
        bad = np.flatnonzero(got[:, 2] != want)
        assert bad.size == 0, f"splat {i}: {bad.size} seeds differ from gps-core's, first k {bad[:5] + k0}"


def test_particle_seeds_equal_gps_core_cluster_scene():
    from gps_pbvr_web_b200 import scenes
    g, sh, deg = PKG.load_ply(scenes.cluster_scene(150_000, seed=0, degree=3))
    W, H = 640, 360
    cam = PKG.OrbitCamera(target=(0.0, 0.0, 0.0), distance=7.0, yaw=0.6, pitch=0.25, up=(0.0, -1.0, 0.0),
                          fov_y=0.9).to_camera(W, H)
    p = PKG.RenderParams(spp_side=1, max_points_per_splat=16384, method=M.Extinction)
    p.pbvr.calibration = Cal.PerSplatFootprint
    p.pbvr.radial_correction = True
    r = PKG.GpsRenderer(W, H, 1)
    try:
        r.set_gaussians_sh(g, sh, deg)
        seed = 77
        r.render_ensembles(cam, p, seed, 1)
        counts = r.debug_counts(0).astype(np.uint64)
        offsets = np.concatenate([[0], np.cumsum(counts)[:-1]])
        nz = np.flatnonzero(counts)
        rng = np.random.default_rng(1)
        picks = {int(nz[0]), int(nz[-1]), int(nz[np.argmax(counts[nz])])} | set(int(x) for x in rng.choice(nz, 12))
        for i in sorted(picks):
            check_splat(r, counts, i, seed, offsets)
    finally:
        r.close()


def test_particle_seeds_above_2_31():
    """136 splats at the cap of 2^24 particles each: the seeds of splats whose particles start above
    2^31 in the ensemble's numbering."""
    from gps_pbvr_web_b200 import scenes
    g, sh, deg = PKG.load_ply(scenes.cluster_scene(20_000, seed=3, degree=0))
    W, H = 320, 180
    cam = PKG.OrbitCamera(target=(0.0, 0.0, 0.0), distance=7.0, yaw=0.6, pitch=0.25, up=(0.0, -1.0, 0.0),
                          fov_y=0.9).to_camera(W, H)
    R = np.asarray(cam.view_rot, np.float64).reshape(3, 3)
    z = (g[:, 0:3].astype(np.float64) - np.asarray(cam.view_pos, np.float64)) @ R[2]
    pick = np.flatnonzero((z > 1.0) & (g[:, 3] > 0.3))[:136]
    p = PKG.RenderParams(spp_side=1, max_points_per_splat=1 << 24, method=M.Extinction, density_scale=1e9)
    p.pbvr.calibration = Cal.PerSplatFootprint
    r = PKG.GpsRenderer(W, H, 1)
    try:
        r.set_gaussians(g[pick].copy())
        r.render_ensembles(cam, p, 5, 1)
        st = r.read_stats()
        counts = r.debug_counts(0).astype(np.uint64)
        total = int(counts.sum())
        assert (1 << 31) < total < (1 << 32) and st.skipped_ensembles == 0, total
        offsets = np.concatenate([[0], np.cumsum(counts)[:-1]])
        high = [i for i in range(len(pick)) if offsets[i] >= (1 << 31)]
        assert len(high) >= 5
        for i in [high[0], high[len(high) // 2], high[-1]]:
            check_splat(r, counts, i, 5, offsets, limit=2048)
    finally:
        r.close()


def _device(which, x):
    xd = torch.from_numpy(np.ascontiguousarray(x, np.float32)).cuda()
    out = torch.empty_like(xd)
    PKG.debug_fmath(which, xd, out)
    torch.cuda.synchronize()
    return out.cpu().numpy()


def _both_forms(which, x):
    a, b = _device(which, x), _device(which | 8, x)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), which  # shared and global tables agree
    return a


def test_device_log_against_libm():
    k = np.arange(1 << 24, dtype=np.float64)
    u = np.maximum((k * 2.0 ** -24).astype(np.float32), np.float32(5.96e-8))  # every Box-Muller u1
    one_minus = (1.0 - (k[1:] * 2.0 ** -24)).astype(np.float32)  # log(1 - c) of the extinction / keep terms
    rng = np.random.default_rng(2)
    wide = np.exp(rng.uniform(np.log(1e-37), np.log(1e37), 1 << 22)).astype(np.float32)
    for x in (u, one_minus, wide):
        got = _both_forms(1, x).astype(np.float64)
        ref = np.log(x.astype(np.float64))
        err = np.abs(got - ref)
        rel = err / np.maximum(np.abs(ref), 1e-30)
        assert np.all((rel <= 4 * 2.0 ** -24) | (err <= 2e-7)), (rel.max(), err.max())
    pos = _both_forms(4, u)
    assert np.array_equal(pos.view(np.uint32), _device(1, u).view(np.uint32))


def test_device_exp_against_libm():
    rng = np.random.default_rng(3)
    x = np.concatenate([np.linspace(-87.0, 88.0, 1 << 22), rng.uniform(-30.0, 0.0, 1 << 22)]).astype(np.float32)
    got = _both_forms(0, x).astype(np.float64)
    ref = np.exp(x.astype(np.float64))
    ulp = np.maximum(np.spacing(np.abs(ref).astype(np.float32)).astype(np.float64), np.finfo(np.float32).tiny)
    assert (np.abs(got - ref) / ulp).max() <= 2.0


def test_device_sin_cos_against_libm():
    k = np.arange(1 << 24, dtype=np.float64)
    th = (np.float32(2.0 * np.pi) * (k * 2.0 ** -24).astype(np.float32)).astype(np.float32)  # every angle 2 pi U
    xd = th.astype(np.float64)
    for which, f in ((2, np.sin), (3, np.cos)):
        err = np.abs(_both_forms(which, th).astype(np.float64) - f(xd))
        assert err.max() <= 2.5e-7, (which, err.max())


def test_device_maths_equal_host_maths():
    """The host form (the O2 mirror's) and the device form give the same bits."""
    rng = np.random.default_rng(4)
    x = np.concatenate([rng.uniform(-90, 90, 1 << 20), np.exp(rng.uniform(-80, 80, 1 << 20))]).astype(np.float32)
    for which in (0, 1, 2, 3):
        xs = np.abs(x) if which == 1 else (np.clip(x, -1e4, 1e4) if which >= 2 else x)
        assert np.array_equal(_device(which, xs).view(np.uint32), O.o2_fmath(which, xs).view(np.uint32)), which
