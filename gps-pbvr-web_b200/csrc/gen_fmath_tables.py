"""Writes fmath_tables.h: the constant tables of the table-driven exp, log and sin/cos in fmath.h.

Every entry is a float32 value given as an exact hexadecimal literal, so the host (the CPU mirror
oracle) and the device (the CUDA kernels) read bit-identical tables. The values come from double-
precision libm evaluations rounded once to float32; exactly representable values (sin and cos at
multiples of pi/2, 2^0, log 1) are written exactly.

  log  : nodes c_i = 1 + i/128, i = -32..64 (mantissas are normalised to [0.75, 1.5)); per node the
         f32 reciprocal r_i = RN(1/c_i) and -log(r_i) split into a float32 high part and residual,
         so log(m) = log1p(m r_i - 1) - log(r_i) holds exactly in real arithmetic.
  exp  : 2^(j/64), j = 0..63, as a float32 high part and residual.
  sincos: (sin, cos)(2 pi j / 256), j = 0..255, each as a float32 high part and residual.

Run: python gps-pbvr-web_b200/csrc/gen_fmath_tables.py   (rewrites the header next to this file)
"""
import math
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def f32(x: float) -> float:
    return float(np.float32(x))


def lit(x: float) -> str:
    x = f32(x)
    if x == 0.0:
        return "0.0f" if math.copysign(1.0, x) > 0 else "-0.0f"
    return float.hex(x) + "f"


def hi_lo(v: float):
    hi = f32(v)
    return hi, f32(v - hi)


def log_table():
    rows = []
    for i in range(-32, 65):
        c = 1.0 + i / 128.0
        r = f32(1.0 / c)
        t = -math.log(r)  # r is exact in double
        th, tl = hi_lo(t)
        rows.append((r, th, tl, 0.0))
    return rows


def exp_table():
    return [hi_lo(2.0 ** (j / 64.0)) for j in range(64)]


def sincos_table():
    rows = []
    for j in range(256):
        q, m = divmod(j, 64)  # quadrant and position inside it: exact zeros and ones at m = 0
        a = 2.0 * math.pi * m / 256.0
        s, c = (0.0, 1.0) if m == 0 else (math.sin(a), math.cos(a))
        for _ in range(q):  # rotate by pi/2: (s, c) -> (c, -s)
            s, c = c, -s
        sh, sl = hi_lo(s)
        ch, cl = hi_lo(c)
        rows.append((sh, ch, sl, cl))
    return rows


def constants():
    ln2 = math.log(2.0)
    k_exp = f32(64.0 / ln2)
    eh, el = hi_lo(ln2 / 64.0)
    k_sc = f32(256.0 / (2.0 * math.pi))
    ph, pl = hi_lo(2.0 * math.pi / 256.0)
    return [("kExpK", k_exp, "64 / ln 2"), ("kExpLHi", eh, "ln 2 / 64, high part"),
            ("kExpLLo", el, "ln 2 / 64 - kExpLHi"), ("kScK", k_sc, "256 / (2 pi)"),
            ("kScPHi", ph, "2 pi / 256, high part"), ("kScPLo", pl, "2 pi / 256 - kScPHi")]


def main():
    lg, ex, sc = log_table(), exp_table(), sincos_table()
    out = ["// Generated by gen_fmath_tables.py: constant tables of the table-driven exp, log and sin/cos",
           "// of fmath.h (exact float32 hexadecimal literals; identical on the host and the device).",
           "#pragma once", "", "namespace gx {", ""]
    for name, v, what in constants():
        out.append(f"constexpr float {name} = {lit(v)};  // {what}")
    out += ["", "constexpr int kLogNodes = 97;   // (1/c_i, -log hi, -log lo, 0), c_i = 1 + i/128, i = -32..64",
            "constexpr int kExpNodes = 64;   // (2^(j/64) hi, lo)",
            "constexpr int kScNodes = 256;   // (sin hi, cos hi, sin lo, cos lo)(2 pi j / 256)", ""]
    for name, rows in [("LOG", lg), ("EXP", ex), ("SC", sc)]:
        out.append(f"#define GX_TAB_{name} \\")
        out.append("    { \\")
        vals = [lit(v) for row in rows for v in row]
        for k in range(0, len(vals), 4):
            out.append("        " + ", ".join(vals[k:k + 4]) + ", \\")
        out.append("    }")
        out.append("")
    out += ["alignas(16) static const float kLogTabH[kLogNodes * 4] = GX_TAB_LOG;",
            "alignas(16) static const float kExpTabH[kExpNodes * 2] = GX_TAB_EXP;",
            "alignas(16) static const float kScTabH[kScNodes * 4] = GX_TAB_SC;",
            "#if defined(__CUDACC__)",
            "static __device__ __align__(16) const float kLogTabD[kLogNodes * 4] = GX_TAB_LOG;",
            "static __device__ __align__(16) const float kExpTabD[kExpNodes * 2] = GX_TAB_EXP;",
            "static __device__ __align__(16) const float kScTabD[kScNodes * 4] = GX_TAB_SC;",
            "#endif", "", "}  // namespace gx", ""]
    with open(os.path.join(HERE, "fmath_tables.h"), "w") as f:
        f.write("\n".join(out))


if __name__ == "__main__":
    main()
