"""The reference's GPU verification phases 2-4 (crates/gps-render/src/verify.rs) restated against
the f64 oracle O1 with the reference's own thresholds, fixed before the first run:
  phase 2: GPS particle and primitive paths vs render_monte_carlo (PSNR >= 60 dB, points within
           4 sigma, no orphans), vs the analytic composite (>= 35 dB, SSIM >= 0.98), identical
           counters between the paths, 3 scan levels, cap truncation, a 4M+-particle splat,
           determinism, history, a 2048x1024x16 frame;
  phase 3: PBVR methods vs render_particles_3d (>= 50 dB, points and candidates within 4 sigma),
           C3+R / ScreenOccupancy / ViewConditioned vs analytic (>= 30 dB), history replay;
  phase 4: SH degrees 0..3 vs eval_sh (>= 60 dB), consecutive degrees differ (< 45 dB).
"""
import math

import numpy as np
import pytest

import oracle as O
from _parity import PKG
from _scenes import BG, cam17, iso, many_70k, scene, to_gpu, verify_scenes

pytestmark = pytest.mark.gpu

W, H, SIDE, SETS = 96, 96, 2, 300
M, Cal, RP = PKG.Method, PKG.Calibration, PKG.RenderPath
SCENES = verify_scenes()


def cam():
    return PKG.OracleCamera()


def image(acc):
    return acc[:, :3].astype(np.float64) / np.maximum(acc[:, 3:4].astype(np.float64), 1.0)


def gpu_mean(items, params, sets, seed0=1, renderer=None, g=None):
    r = renderer or PKG.GpsRenderer(W, H, params.spp_side)
    r.set_gaussians(to_gpu(scene(items)) if g is None else g)
    r.reset_stats()
    r.render_ensembles(cam(), params, seed0, sets)
    acc = r.read_accum()
    st = r.read_stats()
    if renderer is None:
        r.close()
    return acc, st


def params(**kw):
    pb = kw.pop("pbvr", {})
    p = PKG.RenderParams(spp_side=kw.pop("spp_side", SIDE), background=BG, **kw)
    for k, v in pb.items():
        setattr(p.pbvr, k, v)
    return p


# ------------------------------------------------------------------ phase 2
@pytest.mark.parametrize("name,items", SCENES, ids=[s[0] for s in SCENES])
def test_phase2_gps_vs_oracle(name, items):
    ana = O.render_analytic(scene(items), cam17(), W, H, BG)
    seen = []
    for path in [RP.Primitive, RP.Particle]:
        p = params(path=path)
        acc, st = gpu_mean(items, p, SETS)
        gpu = image(acc)
        cpu, cst = O.render_monte_carlo(scene(items), cam17(), W, H, SIDE, SETS, BG, 1,
                                        per_particle_seed=path == RP.Particle, max_points_per_splat=p.max_points_per_splat,
                                        threads=8)
        tol = 4.0 * max(math.sqrt(2.0 * cst["points"]), 1.0)
        assert O.psnr(gpu, cpu) >= 60.0, (path, O.psnr(gpu, cpu))
        assert abs(st.points - cst["points"]) <= tol and st.orphan_subpixels == 0
        assert O.psnr(gpu, ana) >= 35.0 and O.ssim(gpu, ana, W, H) >= 0.98 and st.truncated_splats == 0
        seen.append(st.counters())
    assert seen[0] == seen[1]  # same Poisson stream and cap: identical counters (verify.rs:137-142)


@pytest.mark.parametrize("case", ["70k", "cap50"])
def test_phase2_scan_levels_and_truncation(case):
    if case == "70k":
        sc, p, sets = many_70k(), params(), 8
        g = to_gpu(sc)
    else:
        sc = scene(SCENES[2][1])
        g, p, sets = to_gpu(sc), params(max_points_per_splat=50), 8
    seen = []
    for path in [RP.Primitive, RP.Particle]:
        pp = params(path=path, max_points_per_splat=p.max_points_per_splat)
        acc, st = gpu_mean(None, pp, sets, g=g)
        cpu, cst = O.render_monte_carlo(sc, cam17(), W, H, SIDE, sets, BG, 1, per_particle_seed=path == RP.Particle,
                                        max_points_per_splat=pp.max_points_per_splat, threads=8)
        assert O.psnr(image(acc), cpu) >= 60.0
        assert abs(st.points - cst["points"]) <= 4.0 * max(math.sqrt(2.0 * cst["points"]), 1.0)
        seen.append(st.counters())
    assert seen[0] == seen[1]
    if case == "cap50":
        assert seen[1][1] > 0  # truncated splats are counted, never silent


def test_phase2_four_million_particles_from_one_splat():
    items = [iso(6.0, 0.9, s=0.55)]
    p = params(density_scale=400.0, max_points_per_splat=1 << 24)
    acc, st = gpu_mean(items, p, 2)
    assert st.points > 4_190_000 * 2 * 0.9
    cpu, cst = O.render_monte_carlo(scene(items), cam17(), W, H, SIDE, 2, BG, 1, density_scale=400.0,
                                    per_particle_seed=True, max_points_per_splat=1 << 24, threads=2)
    assert O.psnr(image(acc), cpu) >= 60.0
    assert abs(st.points - cst["points"]) <= 4.0 * math.sqrt(2.0 * cst["points"])


def test_phase2_determinism_and_history():
    items = SCENES[3][1]
    a, _ = gpu_mean(items, params(), 8, 500)
    b, _ = gpu_mean(items, params(), 8, 500)
    c, _ = gpu_mean(items, params(), 8, 600)
    assert np.array_equal(a, b) and not np.array_equal(a, c)
    r = PKG.GpsRenderer(W, H, SIDE)
    acc, _ = gpu_mean(SCENES[1][1], params(), 16, renderer=r)
    assert np.all(np.abs(acc[:, 3] - 16.0) < 1e-3)
    r.reset_accum()
    assert np.all(r.read_accum() == 0.0)
    r.render_ensembles(cam(), params(), 1, 3)
    assert np.all(np.abs(r.read_accum()[:, 3] - 3.0) < 1e-3) and r.accumulated() == 3
    r.close()


def test_phase2_large_frame_2048x1024x16():
    r = PKG.GpsRenderer(2048, 1024, 4)
    r.set_gaussians(to_gpu(scene([iso(6.0, 0.5)])))
    r.reset_stats()
    c = PKG.OracleCamera(focal_x=900.0, focal_y=900.0)
    r.render_ensembles(c, params(spp_side=4), 1, 1)
    acc = r.read_accum()
    assert abs(acc[0, 0] - BG[0]) < 1e-6 and abs(acc[-1, 2] - BG[2]) < 1e-6
    assert abs(acc[512 * 2048 + 1024, 0] - BG[0]) > 1e-3
    assert r.read_stats().orphan_subpixels == 0
    r.close()


# ------------------------------------------------------------------ phase 3
PBVR_CASES = [
    ("Proportional C0", M.Proportional, Cal.None_, False, False, True),
    ("Proportional C3", M.Proportional, Cal.PerSplatFootprint, False, False, True),
    ("Extinction C0", M.Extinction, Cal.None_, False, False, True),
    ("Extinction C1", M.Extinction, Cal.ObjectZoom, False, False, True),
    ("Extinction C2", M.Extinction, Cal.PerSplatDepth, False, False, True),
    ("Extinction C3", M.Extinction, Cal.PerSplatFootprint, False, False, True),
    ("Extinction C3 no-jitter", M.Extinction, Cal.PerSplatFootprint, False, False, False),
    ("Extinction C3 centre-depth", M.Extinction, Cal.PerSplatFootprint, False, True, True),
    ("Extinction C3+R", M.Extinction, Cal.PerSplatFootprint, True, False, True),
    ("Extinction C3+R centre-depth", M.Extinction, Cal.PerSplatFootprint, True, True, True),
]


def pbvr_params(case, **kw):
    _, method, cal, radial, centre, jitter = case
    return params(method=method, max_points_per_splat=1 << 24,
                  pbvr=dict(calibration=cal, radial_correction=radial, centre_depth=centre, low_pass_jitter=jitter), **kw)


@pytest.mark.parametrize("si", [1, 3, 4], ids=[SCENES[i][0] for i in [1, 3, 4]])
@pytest.mark.parametrize("case", PBVR_CASES, ids=[c[0] for c in PBVR_CASES])
def test_phase3_pbvr_vs_oracle(case, si):
    name, items = SCENES[si]
    p = pbvr_params(case)
    acc, st = gpu_mean(items, p, 120)
    gpu = image(acc)
    _, method, cal, radial, centre, jitter = case
    cpu, cst = O.render_particles_3d(scene(items), cam17(), W, H, SIDE, 120, BG, 1, level=int(cal),
                                     rule=0 if method == M.Proportional else 1, radial_correction=radial,
                                     centre_depth=centre, low_pass_jitter=jitter, per_particle_seed=True, threads=8)
    assert O.psnr(gpu, cpu) >= 50.0, O.psnr(gpu, cpu)
    assert abs(st.points - cst["points"]) <= 4.0 * max(math.sqrt(2.0 * cst["points"]), 1.0)
    assert abs(st.candidates - cst["candidates"]) <= 4.0 * max(math.sqrt(2.0 * cst["candidates"]), 1.0)
    assert st.orphan_subpixels == 0 and st.truncated_splats == 0
    if radial:
        ana = O.render_analytic(scene(items), cam17(), W, H, BG)
        assert O.psnr(gpu, ana) >= 30.0


@pytest.mark.parametrize("si", [1, 3, 4])
def test_phase3_screen_occupancy_vs_analytic(si):
    items = SCENES[si][1]
    acc, st = gpu_mean(items, params(method=M.ScreenOccupancy, max_points_per_splat=1), 120)
    ana = O.render_analytic(scene(items), cam17(), W, H, BG)
    bound = len(items) * W * H * SIDE * SIDE * 120
    assert O.psnr(image(acc), ana) >= 30.0 and st.candidates <= bound
    assert st.orphan_subpixels == 0 and st.truncated_splats == 0


@pytest.mark.parametrize("si", [1, 3, 4])
def test_phase3_view_conditioned_matches_gps_counts(si):
    items = SCENES[si][1]
    vp = params(method=M.ViewConditioned, max_points_per_splat=1 << 24, pbvr=dict(calibration=Cal.None_, base_k=4096.0))
    acc, st_vc = gpu_mean(items, vp, 120)
    _, st_gps = gpu_mean(items, params(max_points_per_splat=1 << 24), 120)
    ana = O.render_analytic(scene(items), cam17(), W, H, BG)
    tol = 4.0 * math.sqrt(2.0 * st_gps.points)
    assert O.psnr(image(acc), ana) >= 30.0
    assert abs(st_vc.points - st_gps.points) <= tol and st_vc.undercovered_splats == 0 and st_vc.orphan_subpixels == 0


def test_phase3_70k_c3r_vs_oracle():
    sc = many_70k()
    p = pbvr_params(PBVR_CASES[8])
    acc, st = gpu_mean(None, p, 6, g=to_gpu(sc))
    cpu, cst = O.render_particles_3d(sc, cam17(), W, H, SIDE, 6, BG, 1, radial_correction=True, per_particle_seed=True,
                                     threads=6)
    assert O.psnr(image(acc), cpu) >= 50.0
    assert abs(st.points - cst["points"]) <= 4.0 * math.sqrt(2.0 * cst["points"])


def test_phase3_history_replay_and_offscreen():
    items = SCENES[3][1]
    p = pbvr_params(PBVR_CASES[8])
    r = PKG.GpsRenderer(W, H, SIDE)
    r.set_gaussians(to_gpu(scene(items)))
    r.render_ensembles(cam(), p, 700, 8)
    expected = r.read_accum()
    r.reset_accum()
    r.render_ensembles(cam(), params(), 900, 3)  # GPS history, then PBVR without reloading
    r.reset_accum()
    for seed in range(700, 708):
        r.render_ensembles(cam(), p, seed, 1)
    assert np.array_equal(r.read_accum(), expected)  # batched vs separate
    r.reset_accum()
    off = PKG.OracleCamera(view_pos=np.array([1000.0, 0.0, 0.0]))
    r.render_ensembles(off, p, 800, 2)
    blank = r.read_accum()
    assert np.all(blank[:, 3] == 2.0) and np.all(np.abs(blank[:, :3] - 2.0 * np.array(BG)) < 1e-6)
    moving = pbvr_params(PBVR_CASES[8])
    moving.max_points_per_splat = 16
    r.reset_accum()
    r.render_ensembles(PKG.OracleCamera(view_pos=np.array([0.1, 0.0, 0.0])), moving, 850, 1)
    r.reset_accum()
    for first in [700, 704]:
        r.render_ensembles(cam(), p, first, 4)
    assert np.array_equal(r.read_accum(), expected)
    r.close()


# ------------------------------------------------------------------ phase 4
def _sh_case():
    stride = 15
    s = 99

    def rnd():
        nonlocal s
        s = O.pcg_hash(s)
        return s / 4294967296.0 - 0.5
    dcs, rests, items = [], [], []
    for i in range(4):
        dc = np.array([rnd(), rnd(), rnd()]) * 1.2
        dcs.append(dc)
        rests.append(np.array([rnd() * 0.8 for _ in range(3 * stride)]))
        items.append({"pos": (-0.9 + 0.6 * i, 0.25 * (i - 1.5), 5.0 + 0.7 * i), "log_scale": (math.log(0.22),) * 3,
                      "opacity": 0.85, "color": tuple(dc * 0.28209479177387814 + 0.5)})
    return items, dcs, rests


def test_phase4_sh_degrees_vs_eval_sh():
    items, dcs, rests = _sh_case()
    g = to_gpu(scene(items))
    sh = np.concatenate(rests).astype(np.float32)
    r = PKG.GpsRenderer(W, H, SIDE)
    r.set_gaussians_sh(g, sh, 3)
    images = []
    for deg in range(4):
        cols = []
        for i, it in enumerate(items):
            d = np.asarray(it["pos"]) / np.linalg.norm(it["pos"])
            cols.append(tuple(O.eval_sh(deg, dcs[i], rests[i], d, 15)))
        exp_items = [dict(it, color=cols[i]) for i, it in enumerate(items)]
        r.reset_accum()
        r.render_ensembles(cam(), params(sh_degree=deg), 1, SETS)
        gpu = image(r.read_accum())
        cpu, _ = O.render_monte_carlo(scene(exp_items), cam17(), W, H, SIDE, SETS, BG, 1, per_particle_seed=True, threads=8)
        assert O.psnr(gpu, cpu) >= 60.0, (deg, O.psnr(gpu, cpu))
        images.append(gpu)
    for d in range(1, 4):
        assert O.psnr(images[d], images[d - 1]) < 45.0
    r.set_gaussians(g)  # no SH bands: degree 3 falls back to SH0
    r.reset_accum()
    r.render_ensembles(cam(), params(sh_degree=3), 1, 4)
    assert r.sh_max_degree() == 0 and np.all(np.isfinite(r.read_accum()))
    r.close()


# ------------------------------------------------------------------ launch shapes never change results
@pytest.mark.parametrize("tune", [dict(particle_items=8), dict(particle_items=24), dict(particle_blocks_per_sm=1),
                                  dict(particle_blocks_per_sm=8), dict(ensemble_batch=3)])
def test_tuning_does_not_change_results(tune):
    items = SCENES[4][1]
    for p in [params(), pbvr_params(PBVR_CASES[8]), params(method=M.ScreenOccupancy)]:
        a, sa = gpu_mean(items, p, 10)
        r = PKG.GpsRenderer(W, H, SIDE)
        r.set_tuning(**tune)
        b, sb = gpu_mean(items, p, 10, renderer=r)
        r.close()
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)) and sa.counters() == sb.counters()


@pytest.mark.parametrize("kw", [{"footprint_subpixels": 2, "compensate_blur": True},
                                {"footprint_subpixels": 3},
                                {"adaptive_kappa": 0.6, "footprint_max": 4, "compensate_blur": True}],
                         ids=["fixed2_blur", "fixed3", "adaptive"])
def test_footprint_mode_vs_oracle(kw):
    """The footprint-subpixel Monte-Carlo mode on the GPU against the oracle's render_monte_carlo
    with the same options and the GPU's per-particle seeds (oracle.rs:203-310): PSNR >= 60 dB and
    the same Poisson point counts within 4 sigma, as for plain GPS."""
    from _scenes import layers
    items = layers()
    r = PKG.GpsRenderer(W, H, SIDE)
    r.set_footprint(footprint_subpixels=kw.get("footprint_subpixels", 1), adaptive_kappa=kw.get("adaptive_kappa", 0.0),
                    footprint_max=kw.get("footprint_max", 4), compensate_blur=kw.get("compensate_blur", False))
    p = params()
    acc, st = gpu_mean(items, p, SETS, renderer=r)
    r.close()
    cpu, cst = O.render_monte_carlo(scene(items), cam17(), W, H, SIDE, SETS, BG, 1, per_particle_seed=True,
                                    max_points_per_splat=p.max_points_per_splat, threads=8, **kw)
    gpu = image(acc)
    tol = 4.0 * max(math.sqrt(2.0 * cst["points"]), 1.0)
    assert O.psnr(gpu, cpu) >= 60.0, O.psnr(gpu, cpu)
    assert abs(st.points - cst["points"]) <= tol
    # the footprint really changes the image statistics: fewer points than plain GPS
    plain_acc, plain_st = gpu_mean(items, p, SETS)
    assert st.points < plain_st.points
