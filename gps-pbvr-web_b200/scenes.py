"""Seeded synthetic 3DGS scenes of the benchmark configurations, as binary PLY bytes.

No public dataset is involved: the reference's real capture is not available and not needed;
these generators produce scenes with the stated shapes, sizes and value distributions. The
PLY layout is the one gps-io reads (crates/gps-io/src/lib.rs:265-275): x y z, f_dc_0..2,
f_rest_*, opacity (logit), scale_0..2 (log), rot_0..3 (w x y z). "DC colours uniform in [0,1]"
is read as the linear colour c, stored as f_dc = (c - 0.5) / SH_C0 (the convention of the
reference's tests/gen_synthetic_ply.py).
"""
import math

import numpy as np

SH_C0 = 0.28209479177387814


def _unit_quaternions(rng, n):
    q = rng.normal(size=(n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    return q  # (w, x, y, z)


def _logit(p):
    p = np.clip(p, 1e-7, 1 - 1e-7)
    return np.log(p / (1 - p))


def to_ply(pos, log_scale, rot_wxyz, opacity, dc_colour, sh_rest=None, degree=0) -> bytes:
    """Binary little-endian 3DGS PLY. sh_rest: (n, 3 * ((d+1)^2 - 1)) channel-major."""
    n = pos.shape[0]
    per = (degree + 1) ** 2 - 1 if degree else 0
    names = ["x", "y", "z", "f_dc_0", "f_dc_1", "f_dc_2"] + [f"f_rest_{i}" for i in range(3 * per)] + \
        ["opacity", "scale_0", "scale_1", "scale_2", "rot_0", "rot_1", "rot_2", "rot_3"]
    cols = [pos.astype(np.float32), ((dc_colour - 0.5) / SH_C0).astype(np.float32)]
    if per:
        cols.append(np.asarray(sh_rest, np.float32).reshape(n, 3 * per))
    cols += [_logit(opacity).astype(np.float32).reshape(n, 1), log_scale.astype(np.float32),
             rot_wxyz.astype(np.float32)]
    body = np.ascontiguousarray(np.concatenate(cols, axis=1), dtype="<f4")
    head = "ply\nformat binary_little_endian 1.0\nelement vertex %d\n" % n + \
        "".join(f"property float {c}\n" for c in names) + "end_header\n"
    return head.encode("ascii") + body.tobytes()


def uniform_scene(n=10_000, seed=0):
    """Means U[-1,1]^3, log-scales N(-4, 0.5), uniform rotations, opacity sigmoid(N(0, 1.5)), SH0
    with DC colours U[0,1] (the 10k-Gaussian GPS configuration)."""
    rng = np.random.default_rng(seed)
    pos = rng.uniform(-1.0, 1.0, size=(n, 3))
    log_scale = rng.normal(-4.0, 0.5, size=(n, 3))
    rot = _unit_quaternions(rng, n)
    opacity = 1.0 / (1.0 + np.exp(-rng.normal(0.0, 1.5, size=n)))
    dc = rng.uniform(0.0, 1.0, size=(n, 3))
    return to_ply(pos, log_scale, rot, opacity, dc)


def cluster_scene(n=560_000, seed=0, degree=3, clusters=64):
    """90% of the means from `clusters` anisotropic clusters (centres U[-5,5]^3, per-cluster
    diagonal std U(0.05, 0.8)) and 10% uniform in [-5,5]^3; log-scales N(-3.5, 0.7); uniform
    rotations; opacity sigmoid(N(0.5, 2.0)); SH degree 3 with DC U(0,1) and higher bands N(0, 0.05)."""
    rng = np.random.default_rng(seed)
    n_cl = int(round(0.9 * n))
    centres = rng.uniform(-5.0, 5.0, size=(clusters, 3))
    stds = rng.uniform(0.05, 0.8, size=(clusters, 3))
    which = rng.integers(0, clusters, size=n_cl)
    pos = np.empty((n, 3))
    pos[:n_cl] = centres[which] + rng.normal(size=(n_cl, 3)) * stds[which]
    pos[n_cl:] = rng.uniform(-5.0, 5.0, size=(n - n_cl, 3))
    log_scale = rng.normal(-3.5, 0.7, size=(n, 3))
    rot = _unit_quaternions(rng, n)
    opacity = 1.0 / (1.0 + np.exp(-rng.normal(0.5, 2.0, size=n)))
    dc = rng.uniform(0.0, 1.0, size=(n, 3))
    per = (degree + 1) ** 2 - 1
    rest = rng.normal(0.0, 0.05, size=(n, 3 * per)) if degree else None
    return to_ply(pos, log_scale, rot, opacity, dc, rest, degree)


def orbit_views(distances=(2.5, 7.0, 20.0)):
    """(name, OrbitCamera kwargs) of the near / mid / far views around the origin."""
    names = ("near", "mid", "far")
    return [(names[i] if i < 3 else f"d{d}", dict(target=(0.0, 0.0, 0.0), distance=d, yaw=0.6, pitch=0.25,
                                                    up=(0.0, -1.0, 0.0), fov_y=0.9)) for i, d in enumerate(distances)]


def trajectory(n_cams=16, distance=7.0, pitch=0.25):
    """A 360-degree orbit of n_cams cameras (OrbitCamera kwargs)."""
    return [dict(target=(0.0, 0.0, 0.0), distance=distance, yaw=2.0 * math.pi * k / n_cams, pitch=pitch,
                 up=(0.0, -1.0, 0.0), fov_y=0.9) for k in range(n_cams)]
