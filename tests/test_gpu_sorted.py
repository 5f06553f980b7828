"""Depth-sorted alpha path, demand probe and composite on the GPU (restates
crates/gps-render/src/verify.rs phase 5 and the composite checks of phase 2):
  * the radix sort is bit-exact with a stable sort of the same keys (O2), and a permutation;
  * the blended image is bit-exact with the O2 front-to-back blend and within the reference's
    gate of the analytic composite (PSNR >= 40 dB, SSIM >= 0.99);
  * the demand probe equals the GPS path's mean generated points within 2 %;
  * the RGBA8 composite is bit-exact with O2 and within 1.01 of an 8-bit single-OETF reference.
"""
import math

import numpy as np
import pytest

import oracle as O
from _parity import PKG, lut
from _scenes import BG, cam17, scene, to_gpu, verify_scenes

pytestmark = pytest.mark.gpu
W, H, SIDE = 96, 96, 2


def cam(**kw):
    c = cam17(**kw)
    return PKG.OracleCamera(c[:9].reshape(3, 3), c[9:12], c[12], c[13], c[14], c[15], c[16])


def crowd_items(n=3000):
    s = 4242

    def rnd():
        nonlocal s
        s = O.pcg_hash(s)
        return s / 4294967296.0
    items = []
    for _ in range(n):
        sc = 0.04 + 0.2 * rnd()
        q = np.array([rnd() - 0.5, rnd() - 0.5, rnd() - 0.5, rnd() + 0.2])
        items.append({"pos": (-1.3 + 2.6 * rnd(), -1.3 + 2.6 * rnd(), 4.0 + 5.0 * rnd()),
                      "log_scale": (math.log(sc), math.log(sc * (0.3 + rnd())), math.log(sc * 0.5)),
                      "rot_xyzw": tuple(q / np.linalg.norm(q)), "opacity": 0.2 + 0.7 * rnd(),
                      "color": (rnd(), rnd(), rnd())})
    return items


SCENES = verify_scenes() + [("crowd of 3000", crowd_items())]


def to_image(acc):
    return acc[:, :3].astype(np.float64) / np.maximum(acc[:, 3:4].astype(np.float64), 1.0)


@pytest.mark.parametrize("name,items", SCENES, ids=[s[0] for s in SCENES])
def test_sorted_bit_exact_and_vs_analytic(name, items):
    sc = scene(items)
    g = to_gpu(sc)
    p = PKG.RenderParams(spp_side=SIDE, background=BG)
    r = PKG.GpsRenderer(W, H, SIDE)
    r.set_gaussians(g)
    r.render_sorted(cam(), p, 1)
    acc = r.read_accum()
    keys, vals = r.read_sorted()
    oacc, _, okeys, ovals = O.o2_render_sorted(g, None, 0, lut(), W, H, SIDE, cam().to_array(), p.to_c())
    assert np.array_equal(keys, okeys) and np.array_equal(vals, ovals)
    assert np.all(np.diff(keys.astype(np.int64)) >= 0) and sorted(vals.tolist()) == list(range(len(g)))
    assert np.array_equal(acc.view(np.uint32), oacc.view(np.uint32)), np.abs(acc - oacc).max()
    assert np.all(acc[:, 3] == 1.0) and r.accumulated() == 1
    ana = O.render_analytic(sc, cam17(), W, H, BG)
    img = to_image(acc)
    assert O.psnr(img, ana) >= 40.0 and O.ssim(img, ana, W, H) >= 0.99, (O.psnr(img, ana), O.ssim(img, ana, W, H))
    r.close()


@pytest.mark.parametrize("digit_bits", [4, 6, 8])
def test_radix_sort_300k_is_stable_permutation(digit_bits):
    rng = np.random.default_rng(3)
    n = 300_000
    g = np.zeros((n, 16), np.float32)
    g[:, 0:2] = rng.uniform(-1.3, 1.3, (n, 2))
    g[:, 2] = rng.uniform(4.0, 9.0, n)
    g[:, 3] = 0.5
    g[:, 4:7] = math.log(0.01)
    g[:, 8] = 1.0
    g[:, 12:15] = rng.uniform(0, 1, (n, 3))
    r = PKG.GpsRenderer(W, H, SIDE)
    r.set_gaussians(g)
    r.set_sort_digit_bits(digit_bits)
    p = PKG.RenderParams(spp_side=SIDE)
    r.render_sorted(cam(), p, 1)
    keys, vals = r.read_sorted()
    okeys = np.full(n, 0xFFFFFF, np.uint32)
    _, _, okeys, ovals = O.o2_render_sorted(g, None, 0, lut(), W, H, SIDE, cam().to_array(), p.to_c())
    assert np.array_equal(keys, okeys) and np.array_equal(vals, ovals)
    assert np.count_nonzero(keys != 0xFFFFFF) > 0
    r.close()


def test_demand_probe_matches_gps_points():
    g = to_gpu(scene(crowd_items()))
    p = PKG.RenderParams(spp_side=SIDE, max_points_per_splat=1 << 24)
    r = PKG.GpsRenderer(W, H, SIDE)
    r.set_gaussians(g)
    r.reset_stats()
    r.probe_demand(cam(), p)
    probe = r.read_stats().probe_demand
    r.reset_stats()
    r.render_ensembles(cam(), p, 1, 40)
    points = r.read_stats().points / 40
    rel = abs(probe - points) / max(points, 1.0)
    assert points > 1000 and rel < 0.02, (probe, points)
    r.close()


def test_sorted_after_resize():
    g = to_gpu(scene(crowd_items()))
    r = PKG.GpsRenderer(W, H, SIDE)
    r.resize(64, 64, SIDE)
    r.set_gaussians(g)
    r.render_sorted(cam(), PKG.RenderParams(spp_side=SIDE), 1)
    assert r.read_accum().shape == (64 * 64, 4)
    r.close()


def _srgb(c):
    return np.where(c <= 0.0031308, 12.92 * c, 1.055 * np.power(np.clip(c, 0, None), 1 / 2.4) - 0.055)


@pytest.mark.parametrize("scale", [1, 2])
def test_composite(scale):
    g = to_gpu(scene(verify_scenes()[1][1]))
    p = PKG.RenderParams(spp_side=SIDE, background=BG)
    r = PKG.GpsRenderer(W, H, SIDE)
    r.set_gaussians(g)
    r.render_ensembles(cam(), p, 1, 16)
    acc = r.read_accum()
    out = r.composite(p, W * scale, H * scale)
    ref = O.o2_composite(acc, W, H, p.exposure, p.srgb_output, W * scale, H * scale)
    assert np.array_equal(out, ref)
    # pixel-centred bilinear in linear space, one OETF, 8-bit (verify.rs:241-290)
    ow, oh = W * scale, H * scale
    lin = acc[:, :3].astype(np.float64) / np.maximum(acc[:, 3:4], 1.0)
    lin = lin.reshape(H, W, 3)
    ys, xs = np.mgrid[0:oh, 0:ow]
    qx, qy = (xs + 0.5) / scale - 0.5, (ys + 0.5) / scale - 0.5
    ix, iy = np.floor(qx).astype(int), np.floor(qy).astype(int)
    fx, fy = (qx - ix)[..., None], (qy - iy)[..., None]
    at = lambda y, x: lin[np.clip(y, 0, H - 1), np.clip(x, 0, W - 1)]
    val = (1 - fx) * (1 - fy) * at(iy, ix) + fx * (1 - fy) * at(iy, ix + 1) + (1 - fx) * fy * at(iy + 1, ix) + fx * fy * at(iy + 1, ix + 1)
    expect = _srgb(np.clip(val, 0, 1)) * 255.0
    worst = np.abs(out[:, :3].reshape(oh, ow, 3).astype(np.float64) - expect).max()
    assert worst <= 1.01, worst
    r.close()


@pytest.mark.parametrize("tw,th", [(32, 8), (32, 32)])
def test_blend_tile_shapes_do_not_change_the_image(tw, th):
    g = to_gpu(scene(crowd_items()))
    p = PKG.RenderParams(spp_side=SIDE, background=BG)
    r = PKG.GpsRenderer(W, H, SIDE)
    r.set_gaussians(g)
    r.set_tuning(blend_tile_w=tw, blend_tile_h=th)
    r.render_sorted(cam(), p, 1)
    acc = r.read_accum()
    oacc, _, _, _ = O.o2_render_sorted(g, None, 0, lut(), W, H, SIDE, cam().to_array(), p.to_c())
    assert np.array_equal(acc.view(np.uint32), oacc.view(np.uint32))
    r.close()
