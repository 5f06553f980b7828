"""C-ABI library checks that need no GPU: it loads, exports every function of include/gpsb200.h,
and its host-side pieces (defaults, radius table, cameras, PLY loader) match the reference."""
import ctypes as C
import math
import os
import struct

import numpy as np
import pytest

import oracle as O
from conftest import ROOT, load_package

pkg = load_package()
abi = pkg.abi
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def test_library_exports_every_header_function():
    L = abi.lib()
    names = abi.header_functions()
    assert len(names) >= 40
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    assert set(names) == set(abi.SIGNATURES), set(names) ^ set(abi.SIGNATURES)


def test_params_default_matches_reference():
    # RenderParams::default / PbvrParams::default (crates/gps-render/src/gps.rs:181-228)
    p = abi.ParamsC()
    abi.lib().gpsb_params_default(C.byref(p))
    assert (p.spp_side, p.max_points_per_splat, p.sh_degree, p.path, p.method) == (2, 65536, 3, 1, 0)
    assert abs(p.density_scale - 1.0) < 1e-12 and abs(p.near_z - 0.05) < 1e-7 and p.srgb_output == 1
    assert [round(x, 6) for x in p.background] == [0.05, 0.05, 0.08]
    assert (p.pbvr.calibration, p.pbvr.radial_correction, p.pbvr.centre_depth, p.pbvr.low_pass_jitter) == (3, 0, 0, 1)
    assert p.pbvr.base_k == 512.0 and abs(p.pbvr.reference_pixel_length - 0.01) < 1e-9
    q = pkg.RenderParams().to_c()
    assert bytes(q) == bytes(p)


def test_struct_layouts():
    assert C.sizeof(abi.Gaussian) == 64
    assert C.sizeof(abi.Camera) == 17 * 8
    assert C.sizeof(abi.StatsC) == 13 * 8 + 8


def test_radius_lut_bit_identical_to_oracle():
    a = pkg.radius_lut()
    b = O.radius_lut()
    assert a.shape == (65 * 129,) and np.array_equal(a.view(np.uint32), b.view(np.uint32))


def test_look_at_and_orbit_match_oracle():
    eye, target, up = [3.0, 2.0, -5.0], [0.0, 0.5, 1.0], [0.0, 1.0, 0.0]
    c = pkg.OracleCamera.look_at(eye, target, up, 0.9, 128, 96).to_array()
    assert np.allclose(c, O.look_at(eye, target, up, 0.9, 128, 96), rtol=0, atol=1e-12)
    cam = pkg.OrbitCamera(target=(1.0, 2.0, 3.0), distance=7.0, yaw=0.7, pitch=0.3).to_camera(64, 48)
    e = O.orbit_eye([1.0, 2.0, 3.0], 7.0, 0.7, 0.3, [0, 1.0, 0])
    assert np.allclose(cam.view_pos, e, atol=1e-12)
    t = cam.view_rot @ (np.array([1.0, 2.0, 3.0]) - cam.view_pos)
    assert abs(t[0]) < 1e-9 and abs(t[1]) < 1e-9 and abs(t[2] - 7.0) < 1e-9


def test_estimate_memory():
    # crates/gps-render/src/gps.rs:1105-1110: 1920x1080, S=4 is ~95 MiB
    m = pkg.estimate_memory(1920, 1080, 2, 0)
    assert m["depth_winner_bytes"] + m["accum_bytes"] == 8 * 1920 * 1080 * 4 + 16 * 1920 * 1080
    assert abs((m["depth_winner_bytes"] + m["accum_bytes"]) / 1048576.0 - 95.0) < 1.0


def test_create_without_device_reports_an_error():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(pkg.GpsError) as e:
        pkg.GpsRenderer(64, 64, 1)
    assert "device" in str(e.value).lower() or "cuda" in str(e.value).lower()


# ----------------------------------------------------------------- PLY (crates/gps-io/src/lib.rs:376-458)
def _header(fmt, n, sh1):
    h = f"ply\nformat {fmt} 1.0\nelement vertex {n}\n"
    for p in ["x", "y", "z", "f_dc_0", "f_dc_1", "f_dc_2"]:
        h += f"property float {p}\n"
    if sh1:
        for i in range(9):
            h += f"property float f_rest_{i}\n"
    for p in ["opacity", "scale_0", "scale_1", "scale_2", "rot_0", "rot_1", "rot_2", "rot_3"]:
        h += f"property float {p}\n"
    return h + "end_header\n"


def test_ply_binary_roundtrip_sh1():
    b = _header("binary_little_endian", 2, True).encode()
    for v in range(2):
        b += struct.pack("<23f", *[(v * 100 + k) * 0.01 for k in range(23)])
    g, sh, d = pkg.load_ply(b)
    assert (g.shape[0], d) == (2, 1) and sh.size == 18
    assert np.allclose(g[1, :3], [1.0, 1.01, 1.02])
    # opacity follows f_rest_8 (index 15): activated = sigmoid(0.15)
    assert abs(g[0, 3] - 1 / (1 + math.exp(-0.15))) < 1e-6
    assert abs(g[0, 8] - 0.19) < 1e-6  # rot_0 = w
    assert abs(g[0, 12] - (0.03 * 0.28209479177387814 + 0.5)) < 1e-6  # colour = f_dc * C0 + 0.5


def test_ply_ascii_and_activation():
    s = _header("ascii", 1, False) + "1 2 3  0.5 0 0  0  0 0 0  1 0 0 0\n"
    g, sh, d = pkg.load_ply(s.encode())
    assert abs(g[0, 3] - 0.5) < 1e-7 and list(g[0, 8:12]) == [1, 0, 0, 0] and d == 0


@pytest.mark.parametrize("data,needle", [
    (b"hello", "no end_header"),
    (b"nope\nend_header\n", "not a PLY"),
    (_header("binary_little_endian", 5, False).encode() + b"\0" * 10, "truncated"),
    (_header("binary_little_endian", 200_000_001, False).encode(), "exceeds limit"),
    ((_header("ascii", 1, False) + "nan 0 0 0 0 0 0 0 0 0 0 0 0 0\n").encode(), "non-finite"),
    (b"ply\nformat ascii 1.0\nelement vertex 0\nproperty float x\nend_header\n", "missing required property 'y'"),
])
def test_ply_rejects_bad_input(data, needle):
    with pytest.raises(pkg.GpsError) as e:
        pkg.load_ply(data)
    assert needle in str(e.value)


def test_ply_bad_sh_count():
    h = "ply\nformat ascii 1.0\nelement vertex 0\n"
    for p in ["x", "y", "z", "f_dc_0", "f_dc_1", "f_dc_2", "opacity", "scale_0", "scale_1", "scale_2", "rot_0",
              "rot_1", "rot_2", "rot_3", "f_rest_0"]:
        h += f"property float {p}\n"
    with pytest.raises(pkg.GpsError) as e:
        pkg.load_ply((h + "end_header\n").encode())
    assert "1 f_rest_* properties" in str(e.value)


def test_ply_huge_count_rejected_before_allocation():
    for fmt in ["binary_little_endian", "ascii"]:
        b = _header(fmt, 200_000_000, False).encode() + b"1 2 3\n"
        with pytest.raises(pkg.GpsError) as e:
            pkg.load_ply(b)
        assert "truncated" in str(e.value)


def test_ply_fixture_synthetic_sh1():
    data = open(os.path.join(GOLDEN, "synthetic_sh1.ply"), "rb").read()
    g, sh, d = pkg.load_ply(data)
    assert g.shape == (400, 16) and d == 1 and sh.size == 400 * 9
    assert np.all((g[:, 3] > 0) & (g[:, 3] < 1))
    assert np.allclose(g[:220, 5], math.log(0.02), atol=1e-6)  # ground disk scale_1


def test_scene_generators_roundtrip():
    from gps_pbvr_web_b200 import scenes
    g, sh, d = pkg.load_ply(scenes.uniform_scene(1000, seed=0))
    assert g.shape == (1000, 16) and d == 0
    assert np.all(np.abs(g[:, :3]) <= 1.0) and np.all((g[:, 12:15] > -1e-5) & (g[:, 12:15] < 1 + 1e-5))
    g, sh, d = pkg.load_ply(scenes.cluster_scene(2000, seed=1, degree=3))
    assert g.shape == (2000, 16) and d == 3 and sh.size == 2000 * 45
