"""Scenes of the reference's own tests, as f64 dicts (crates/gps-core/tests/*.rs, verify.rs:18-39)."""
import math

import numpy as np

BG = (0.05, 0.05, 0.08)


def scene(items):
    """items: list of dicts with pos, log_scale, rot_xyzw, opacity, color."""
    return {
        "pos": np.array([g["pos"] for g in items], dtype=np.float64).reshape(-1, 3),
        "log_scale": np.array([g["log_scale"] for g in items], dtype=np.float64).reshape(-1, 3),
        "rot_xyzw": np.array([g.get("rot_xyzw", (0.0, 0.0, 0.0, 1.0)) for g in items], dtype=np.float64).reshape(-1, 4),
        "opacity": np.array([g["opacity"] for g in items], dtype=np.float64),
        "color": np.array([g["color"] for g in items], dtype=np.float64).reshape(-1, 3),
    }


def iso(z, o, col=(0.9, 0.4, 0.2), x=0.0, s=0.15):
    return {"pos": (x, 0.0, z), "log_scale": (math.log(s),) * 3, "opacity": o, "color": col}


def quat_normalize(q):
    q = np.asarray(q, dtype=np.float64)
    return tuple(q * (1.0 / math.sqrt(float(np.dot(q, q)))))


def aniso(z=6.0, x=0.0, y=0.0):
    return {"pos": (x, y, z), "log_scale": (math.log(0.28), math.log(0.10), math.log(0.06)),
            "rot_xyzw": quat_normalize((0.20, -0.45, 0.30, 0.82)), "opacity": 0.7, "color": (0.3, 0.5, 0.95)}


def layers():
    # crates/gps-core/tests/cpp_crosscheck.rs:27-35
    return [iso(9.0, 0.8, (0.15, 0.7, 0.25), 0.1), iso(5.0, 0.6, (0.9, 0.2, 0.2), -0.1), iso(7.0, 0.4, (0.2, 0.3, 0.9), 0.0)]


def cam17(focal=200.0, pos=(0.0, 0.0, 0.0), cx=0.0, cy=0.0, low_pass=0.3, rot=None):
    """OracleCamera (crates/gps-core/src/oracle.rs:44-48) as 17 doubles (gpsb_camera layout)."""
    r = np.eye(3) if rot is None else np.asarray(rot, dtype=np.float64)
    return np.concatenate([r.reshape(-1), np.asarray(pos, dtype=np.float64), [focal, focal, cx, cy, low_pass]])


def verify_scenes():
    """verify.rs:21-39: name -> list of splats."""
    c = (0.9, 0.4, 0.2)
    return [
        ("single o=0.1", [iso(6.0, 0.1, c)]),
        ("single o=0.5", [iso(6.0, 0.5, c)]),
        ("single o=0.9", [iso(6.0, 0.9, c)]),
        ("front/back", [iso(9.0, 0.8, (0.15, 0.7, 0.25)), iso(5.0, 0.6, (0.9, 0.2, 0.2))]),
        ("anisotropic", [aniso()]),
    ]


def to_gpu(sc):
    """GpuGaussian::from_oracle (crates/gps-render/src/gps.rs:51-58): (n, 16) f32."""
    n = len(sc["opacity"])
    g = np.zeros((n, 16), dtype=np.float32)
    g[:, 0:3] = sc["pos"]
    g[:, 3] = sc["opacity"]
    g[:, 4:7] = sc["log_scale"]
    q = sc["rot_xyzw"]
    g[:, 8] = q[:, 3]
    g[:, 9:12] = q[:, 0:3]
    g[:, 12:15] = sc["color"]
    return g


def many_70k():
    """70,000 tiny splats (verify.rs:174-184)."""
    i = np.arange(70_000, dtype=np.int64)
    gx = (i % 280) / 280.0 - 0.5
    gy = (i // 280) / 250.0 - 0.5
    pos = np.stack([gx * 0.9, gy * 0.9, 6.0 + (i % 7) * 0.1], axis=1)
    op = 0.3 + 0.6 * ((i * 37 % 100) / 100.0)
    col = np.stack([(i % 5) / 5.0, (i % 3) / 3.0, np.full(len(i), 0.5)], axis=1)
    return {"pos": pos, "log_scale": np.full((len(i), 3), math.log(0.012)), "rot_xyzw": np.tile([0, 0, 0, 1.0], (len(i), 1)),
            "opacity": op, "color": col}
