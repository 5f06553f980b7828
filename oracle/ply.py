"""PLY reader of the oracle. TEST INFRASTRUCTURE ONLY.

A numpy restatement of gps-io's `load_ply` for binary little-endian 3DGS files with float
properties (crates/gps-io/src/lib.rs:260-373: property lookup by name, f_rest_0.. counted up to the
first gap, SH degree from the rest count, body length checked against the vertex count, every
value finite) followed by `Gaussians::activated` (lib.rs:84-96: opacity = sigmoid(logit) in f64,
log-scale kept, rotation (w, x, y, z) cast as read) and `GpuGaussian::from_activated`
(crates/gps-render/src/gps.rs:41-49: linear colour f_dc * SH_C0 + 0.5 in f64, every field rounded
once to f32). It lets the CPU baseline and the CPU tests read the synthetic scenes without the
renderer library; the renderer's own loader (gps-pbvr-web_b200/csrc/ply.cpp) is checked against it.
"""
import math

import numpy as np

SH_C0 = 0.28209479177387814  # crates/gps-core/src/lib.rs


def _sigmoid(x):
    # gps_core::sigmoid (crates/gps-core/src/lib.rs:21-23) with the C library's exp, element by element
    return np.array([1.0 / (1.0 + math.exp(-float(v))) for v in x], dtype=np.float64)


def read_ply(data: bytes):
    """Returns (splats (n, 16) f32 in the 64-byte record layout, sh_rest (n, 3 * per) f32
    channel-major or None, degree, f64 scene dict of the O1 renderers made from the f32 records)."""
    end = data.find(b"end_header\n")
    if not data.startswith(b"ply\n") or end < 0:
        raise ValueError("not a PLY file")
    head = data[:end].decode("ascii").split("\n")
    if "format binary_little_endian 1.0" not in head:
        raise ValueError("only binary little-endian PLY is read here")
    n = None
    props = []
    for line in head:
        t = line.split()
        if t[:2] == ["element", "vertex"]:
            n = int(t[2])
        elif t[:1] == ["property"]:
            if t[1] != "float":
                raise ValueError(f"property {t[-1]}: only float properties are read here")
            props.append(t[2])
    if n is None:
        raise ValueError("no vertex element")
    body = data[end + len(b"end_header\n"):]
    stride = 4 * len(props)
    if len(body) < n * stride:
        raise ValueError(f"truncated: expected {n * stride} bytes, got {len(body)}")
    a = np.frombuffer(body[:n * stride], dtype="<f4").reshape(n, len(props))
    col = {name: k for k, name in enumerate(props)}
    rest = []
    while f"f_rest_{len(rest)}" in col:
        rest.append(col[f"f_rest_{len(rest)}"])
    degree = {0: 0, 9: 1, 24: 2, 45: 3}.get(len(rest))
    if degree is None:
        raise ValueError(f"{len(rest)} f_rest properties do not form an SH degree")
    need = ["x", "y", "z", "f_dc_0", "f_dc_1", "f_dc_2", "opacity", "scale_0", "scale_1", "scale_2",
            "rot_0", "rot_1", "rot_2", "rot_3"]
    for name in need:
        if name not in col:
            raise ValueError(f"missing property {name}")
    used = a[:, [col[k] for k in need] + rest]
    if not np.isfinite(used).all():
        raise ValueError("non-finite value")
    pos = a[:, [col["x"], col["y"], col["z"]]].astype(np.float64)
    dc = a[:, [col["f_dc_0"], col["f_dc_1"], col["f_dc_2"]]].astype(np.float64)
    op = _sigmoid(a[:, col["opacity"]])
    ls = a[:, [col["scale_0"], col["scale_1"], col["scale_2"]]].astype(np.float64)
    q = a[:, [col["rot_0"], col["rot_1"], col["rot_2"], col["rot_3"]]].astype(np.float64)  # w x y z
    colour = dc * SH_C0 + 0.5
    g = np.zeros((n, 16), np.float32)
    g[:, 0:3] = pos
    g[:, 3] = op
    g[:, 4:7] = ls
    g[:, 8:12] = q
    g[:, 12:15] = colour
    sh = np.ascontiguousarray(a[:, rest], dtype=np.float32) if rest else None
    return g, sh, degree, o1_scene(g)


def o1_scene(g):
    """The f64 scene dict of the O1 renderers from (n, 16) f32 records (the values the GPU sees)."""
    return {"pos": g[:, 0:3].astype(np.float64), "log_scale": g[:, 4:7].astype(np.float64),
            "rot_xyzw": np.concatenate([g[:, 9:12], g[:, 8:9]], axis=1).astype(np.float64),
            "opacity": g[:, 3].astype(np.float64), "color": g[:, 12:15].astype(np.float64)}
