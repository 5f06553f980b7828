"""ctypes bindings of the oracle library. TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import this package; the
renderer never does. O1 = f64 restatement of crates/gps-core (the semantic oracle and the timed
CPU baseline). O2 = f32 mirror of shaders/gps_splat.wgsl (the bit-exact target of the CUDA
kernels). See oracle/o1_core.cpp and oracle/o2_mirror.cpp for the citations.
"""
import ctypes as C
import os

import numpy as np

from . import build as _build

_lib = None


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libgpsoracle.so")
        _build.build()  # no-op when the library is up to date
        _lib = C.CDLL(path)
        _declare(_lib)
    return _lib


P = C.c_void_p
D = C.c_double
U32 = C.c_uint32
SZ = C.c_size_t


def _declare(L):
    for name, res, args in [
        ("o1_dilog", D, [D]), ("o1_inv_dilog", D, [D]), ("o1_sigmoid", D, [D]),
        ("o1_expected_point_count", D, [D, D]), ("o1_pcg_hash", U32, [U32]),
        ("o1_particle_seed", U32, [C.c_int, U32, U32, U32]), ("o1_ordered_depth_key", U32, [C.c_float]),
        ("o1_ordered_depth_key_inverse", C.c_float, [U32]), ("o1_sample_corrected_radius", D, [D, D]),
        ("o1_radial_keep_probability", D, [D, D]), ("o1_calibrated_count", D, [C.c_int, C.c_int, D, D, D, P]),
        ("o1_radius_lut", None, [P]), ("o1_radius_from_lut", D, [P, D, D]),
        ("o1_poisson_stream", None, [D, U32, P, SZ]), ("o1_covariance_2d", None, [P, P, P, D, D, D, D, P]),
        ("o1_eval_sh", None, [C.c_int, P, P, P, C.c_int, P]),
        ("o1_render_analytic", None, [P, SZ, P, SZ, SZ, P, P]),
        ("o1_render_monte_carlo", None, [P, SZ, P, SZ, SZ, SZ, SZ, P, U32, P, P, P, C.c_int]),
        ("o1_render_particles_3d", None, [P, SZ, P, SZ, SZ, SZ, SZ, P, U32, P, P, P, C.c_int]),
        ("o1_psnr", D, [P, P, SZ]), ("o1_ssim", D, [P, P, SZ, SZ]),
        ("o1_look_at", None, [P, P, P, D, U32, U32, P]), ("o1_orbit_eye", None, [P, D, D, D, P, P]),
        ("o2_render_ensembles", C.c_int, [P, U32, P, U32, P, U32, U32, U32, P, P, U32, U32, P, P, P, P]),
        ("o2_render_ensembles_mt", C.c_int, [P, U32, P, U32, P, U32, U32, U32, P, P, U32, U32, P, P, P, P, U32]),
        ("o2_render_sorted", C.c_int, [P, U32, P, U32, P, U32, U32, U32, P, P, P, P, P, P]),
        ("o2_composite", C.c_int, [P, U32, U32, C.c_float, U32, U32, U32, P]),
        ("o2_fmath_eval", None, [C.c_int, P, P, SZ]),
        ("o2_fast_check", C.c_int, [P, U32, P, U32, P, U32, U32, U32, P, P, U32, U32, U32, C.c_int, P]),
    ]:
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _f64(x, n=None):
    a = np.ascontiguousarray(np.asarray(x, dtype=np.float64))
    if n is not None:
        assert a.size == n
    return a


# ------------------------------------------------------------------ O1 scalar maths
def dilog(x): return lib().o1_dilog(x)
def inv_dilog(x): return lib().o1_inv_dilog(x)
def sigmoid(x): return lib().o1_sigmoid(x)
def expected_point_count(det, o): return lib().o1_expected_point_count(det, o)
def pcg_hash(v): return lib().o1_pcg_hash(v)
def particle_seed(frame_varying, s, k, f): return lib().o1_particle_seed(int(frame_varying), s, k, f)
def ordered_depth_key(d): return lib().o1_ordered_depth_key(d)
def ordered_depth_key_inverse(k): return lib().o1_ordered_depth_key_inverse(k)
def sample_corrected_radius(o, u): return lib().o1_sample_corrected_radius(o, u)
def radial_keep_probability(o, r2): return lib().o1_radial_keep_probability(o, r2)


def calibrated_count(level, rule, o, base_k, density, object_depth=0.0, splat_depth=0.0, fx=1.0, fy=1.0,
                     near_z=0.0, refl=0.01, footprint_area=0.0, spp=1.0):
    a = _f64([object_depth, splat_depth, fx, fy, near_z, refl, footprint_area, spp])
    return lib().o1_calibrated_count(level, rule, o, base_k, density, _p(a))


def radius_lut():
    t = np.zeros(65 * 129, dtype=np.float32)
    lib().o1_radius_lut(_p(t))
    return t


def radius_from_lut(lut, o, u):
    lut = np.ascontiguousarray(lut, dtype=np.float32)
    return lib().o1_radius_from_lut(_p(lut), o, u)


def poisson_stream(lam, seed, n):
    out = np.zeros(n, dtype=np.int32)
    lib().o1_poisson_stream(lam, seed, _p(out), n)
    return out


def covariance_2d(log_scale, rot_xyzw, mean, fx, fy, tan_fov, low_pass):
    out = np.zeros(4)
    lib().o1_covariance_2d(_p(_f64(log_scale)), _p(_f64(rot_xyzw)), _p(_f64(mean)), fx, fy, tan_fov, low_pass, _p(out))
    return out  # column-major (xx, xy, yx, yy)


def eval_sh(degree, dc, rest, direction, stride):
    out = np.zeros(3)
    r = None if rest is None else _f64(rest)
    lib().o1_eval_sh(degree, _p(_f64(dc)), _p(r), _p(_f64(direction)), stride, _p(out))
    return out


# ------------------------------------------------------------------ O1 renderers
def _scene14(scene):
    """scene: dict of f64 arrays pos (n,3), log_scale (n,3), rot_xyzw (n,4), opacity (n,), color (n,3)."""
    n = len(scene["opacity"])
    a = np.zeros((n, 14))
    a[:, 0:3] = scene["pos"]
    a[:, 3:6] = scene["log_scale"]
    a[:, 6:10] = scene["rot_xyzw"]
    a[:, 10] = scene["opacity"]
    a[:, 11:14] = scene["color"]
    return np.ascontiguousarray(a), n


def render_analytic(scene, cam17, w, h, bg):
    s, n = _scene14(scene)
    img = np.zeros((h * w, 3))
    lib().o1_render_analytic(_p(s), n, _p(_f64(cam17, 17)), w, h, _p(_f64(bg, 3)), _p(img))
    return img


def render_monte_carlo(scene, cam17, w, h, spp_side, sets, bg, seed, footprint_subpixels=1, adaptive_kappa=0.0,
                       footprint_max=4, compensate_blur=False, density_scale=1.0, per_particle_seed=False,
                       max_points_per_splat=0xFFFFFFFF, threads=1):
    s, n = _scene14(scene)
    img = np.zeros((h * w, 3))
    st = np.zeros(3)
    opt = _f64([footprint_subpixels, adaptive_kappa, footprint_max, float(compensate_blur), density_scale,
                float(per_particle_seed), float(max_points_per_splat)])
    lib().o1_render_monte_carlo(_p(s), n, _p(_f64(cam17, 17)), w, h, spp_side, sets, _p(_f64(bg, 3)), seed, _p(opt),
                                _p(img), _p(st), threads)
    return img, {"points": st[0], "candidates": st[1], "subpixel_writes": st[2]}


def render_particles_3d(scene, cam17, w, h, spp_side, sets, bg, seed, level=3, rule=1, radial_correction=False,
                        base_k=512.0, reference_pixel_length=0.01, near_z=0.05, low_pass_jitter=True,
                        centre_depth=False, linearized_projection=False, density_scale=1.0, per_particle_seed=False,
                        threads=1, max_points_per_splat=0xFFFFFFFF):
    """rule: 0 Proportional, 1 Extinction, 2 Dilog (crates/gps-core/src/lib.rs:296-300)."""
    s, n = _scene14(scene)
    img = np.zeros((h * w, 3))
    st = np.zeros(3)
    opt = _f64([level, rule, float(radial_correction), base_k, reference_pixel_length, near_z, float(low_pass_jitter),
                float(centre_depth), float(linearized_projection), density_scale, float(per_particle_seed),
                float(max_points_per_splat)])
    lib().o1_render_particles_3d(_p(s), n, _p(_f64(cam17, 17)), w, h, spp_side, sets, _p(_f64(bg, 3)), seed, _p(opt),
                                 _p(img), _p(st), threads)
    return img, {"points": st[0], "candidates": st[1], "subpixel_writes": st[2]}


def psnr(a, b):
    a = _f64(a).reshape(-1, 3)
    b = _f64(b).reshape(-1, 3)
    return lib().o1_psnr(_p(a), _p(b), min(len(a), len(b)))


def ssim(a, b, w, h):
    a = _f64(a).reshape(-1, 3)
    b = _f64(b).reshape(-1, 3)
    return lib().o1_ssim(_p(a), _p(b), w, h)


def look_at(eye, target, up, fov_y, w, h):
    out = np.zeros(17)
    lib().o1_look_at(_p(_f64(eye)), _p(_f64(target)), _p(_f64(up)), fov_y, w, h, _p(out))
    return out


def orbit_eye(target, distance, yaw, pitch, up):
    out = np.zeros(3)
    lib().o1_orbit_eye(_p(_f64(target)), distance, yaw, pitch, _p(_f64(up)), _p(out))
    return out


# ------------------------------------------------------------------ O2 mirror
def _o2_scene(splats, sh):
    g = np.ascontiguousarray(splats, dtype=np.float32).reshape(-1, 16)
    s = None if sh is None else np.ascontiguousarray(sh, dtype=np.float32)
    return g, s


def o2_render_ensembles(splats, sh, sh_degree, lut, w, h, spp_side, cam17, params, first_seed, count, accum=None,
                        stats=None, want_counts=False, want_packed=False, threads=1):
    """Returns (accum (h*w,4) f32, stats (12,) u64, counts (count,n) u32 | None, packed (count,h*w*S) u64 | None).
    threads > 1 splits every stage over host threads (winners by a packed 64-bit minimum); the
    results equal the sequential form's."""
    import ctypes
    g, s = _o2_scene(splats, sh)
    n = g.shape[0]
    side = max(1, min(int(spp_side), 4))
    S = side * side
    acc = np.zeros((h * w, 4), np.float32) if accum is None else np.ascontiguousarray(accum, np.float32).copy()
    st = np.zeros(12, np.uint64) if stats is None else np.ascontiguousarray(stats, np.uint64).copy()
    counts = np.zeros((count, n), np.uint32) if want_counts else None
    packed = np.zeros((count, h * w * S), np.uint64) if want_packed else None
    lut = np.ascontiguousarray(lut, np.float32)
    lib().o2_render_ensembles_mt(_p(g), n, _p(s), sh_degree, _p(lut), w, h, side, _p(_f64(cam17, 17)),
                                 ctypes.cast(ctypes.pointer(params), C.c_void_p), first_seed, count, _p(acc), _p(st),
                                 _p(counts), _p(packed), max(1, int(threads)))
    return acc, st, counts, packed


def o2_fast_check(splats, sh, sh_degree, lut, w, h, spp_side, cam17, params, first_seed, count, perturb_seed=0,
                  mode=0):
    """The renderer's PBVR fast decisions restated with every approximation pushed to the edge of
    its assumed error bound (mode 0 random signs, 1 all +, 2 all -), against the exact path over
    every particle: returns (particles, decided, decided wrongly, points)."""
    import ctypes
    g, s = _o2_scene(splats, sh)
    out = np.zeros(4, np.uint64)
    rc = lib().o2_fast_check(_p(g), g.shape[0], _p(s), sh_degree, _p(np.ascontiguousarray(lut, np.float32)), w, h,
                             spp_side, _p(_f64(cam17, 17)), ctypes.cast(ctypes.pointer(params), C.c_void_p),
                             first_seed, count, perturb_seed, mode, _p(out))
    if rc != 0:
        raise ValueError("o2_fast_check: PBVR methods only")
    return tuple(int(v) for v in out)


def o2_render_sorted(splats, sh, sh_degree, lut, w, h, spp_side, cam17, params):
    import ctypes
    g, s = _o2_scene(splats, sh)
    n = g.shape[0]
    acc = np.zeros((h * w, 4), np.float32)
    st = np.zeros(12, np.uint64)
    keys = np.zeros(n, np.uint32)
    vals = np.zeros(n, np.uint32)
    lib().o2_render_sorted(_p(g), n, _p(s), sh_degree, _p(np.ascontiguousarray(lut, np.float32)), w, h, spp_side,
                           _p(_f64(cam17, 17)), ctypes.cast(ctypes.pointer(params), C.c_void_p), _p(acc), _p(st),
                           _p(keys), _p(vals))
    return acc, st, keys, vals


def o2_composite(accum, w, h, exposure, gamma_on, out_w, out_h):
    acc = np.ascontiguousarray(accum, np.float32).reshape(-1, 4)
    out = np.zeros((out_h * out_w, 4), np.uint8)
    lib().o2_composite(_p(acc), w, h, exposure, int(gamma_on), out_w, out_h, _p(out))
    return out


def o2_fmath(which, x):
    """which: 0 exp, 1 log, 2 sin, 3 cos, 4 pow(x, 1/2.4), 5 log for positive normal arguments."""
    x = np.ascontiguousarray(x, np.float32)
    out = np.zeros_like(x)
    lib().o2_fmath_eval(which, _p(x), _p(out), x.size)
    return out
