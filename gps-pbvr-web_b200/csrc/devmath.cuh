// Device maths shared by the particle-path and sorted-path kernels: projection, Li2 and its
// inverse, the radius table lookup, Poisson sampling and the SH colour, each following
// shaders/gps_splat.wgsl expression by expression (compile with --fmad=false).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "internal.h"

#define F_(x) ((float)(x))

namespace gpsb {
using gx::clamp_;
using gx::div_;
using gx::f2b;
using gx::f2u;
using gx::fmax_;
using gx::fmin_;
using gx::sqrt_;

// ----------------------------------------------------------------------------- shared maths
// Bases of the fmath tables (log, exp, sin/cos) a kernel reads: shared-memory copies in the
// particle kernel, the global copies elsewhere; both hold the same values.
struct FTabs {
    const float* lg;
    const float* ex;
    const float* sc;
};
constexpr int kTabFloats = gx::kScNodes * 4 + gx::kLogNodes * 4 + gx::kExpNodes * 2;  // staged table floats

// Copies the tables into shared memory at s (16-byte aligned, kTabFloats floats) and returns
// their bases; the caller synchronises the block before the first use.
__device__ __forceinline__ FTabs stage_tabs(float* s) {
    for (int k = threadIdx.x; k < kTabFloats; k += blockDim.x) {
        float v;
        if (k < gx::kScNodes * 4) v = gx::kScTabD[k];
        else if (k < gx::kScNodes * 4 + gx::kLogNodes * 4) v = gx::kLogTabD[k - gx::kScNodes * 4];
        else v = gx::kExpTabD[k - gx::kScNodes * 4 - gx::kLogNodes * 4];
        s[k] = v;
    }
    return FTabs{s + gx::kScNodes * 4, s + gx::kScNodes * 4 + gx::kLogNodes * 4, s};
}
struct Proj {
    bool ok;
    float mx, my, a, b, c, depth;
};

__device__ __forceinline__ float dot3(float ax, float ay, float az, float bx, float by, float bz) {
    return ax * bx + ay * by + az * bz;
}

__device__ __forceinline__ void rot_cols(float4 q, float* c0, float* c1, float* c2) {
    float len = sqrt_(q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w);
    float w = div_(q.x, len), x = div_(q.y, len), y = div_(q.z, len), z = div_(q.w, len);
    c0[0] = F_(1.0) - F_(2.0) * (y * y + z * z);
    c0[1] = F_(2.0) * (x * y + w * z);
    c0[2] = F_(2.0) * (x * z - w * y);
    c1[0] = F_(2.0) * (x * y - w * z);
    c1[1] = F_(1.0) - F_(2.0) * (x * x + z * z);
    c1[2] = F_(2.0) * (y * z + w * x);
    c2[0] = F_(2.0) * (x * z + w * y);
    c2[1] = F_(2.0) * (y * z - w * x);
    c2[2] = F_(1.0) - F_(2.0) * (x * x + y * y);
}

// project (gps_splat.wgsl:165-206)
__device__ inline Proj project(const FrameConst& f, float4 g0, float4 g1, float4 g2) {
    Proj pr;
    pr.ok = false;
    float px = g0.x - f.pos[0], py = g0.y - f.pos[1], pz = g0.z - f.pos[2];
    float cx = dot3(f.rot0[0], f.rot0[1], f.rot0[2], px, py, pz);
    float cy = dot3(f.rot1[0], f.rot1[1], f.rot1[2], px, py, pz);
    float cz = dot3(f.rot2[0], f.rot2[1], f.rot2[2], px, py, pz);
    if (cz <= fmax_(f.near_z, F_(1e-4))) return pr;
    float lim = gxc::kFrustumLim;
    float tx = clamp_(div_(cx, cz), -lim, lim) * cz;
    float ty = clamp_(div_(cy, cz), -lim, lim) * cz;
    float fx = f.fx, fy = f.fy;
    float iz = div_(F_(1.0), cz);
    float s0 = fx * iz, s1 = -fx * tx * iz * iz;
    float s2 = fy * iz, s3 = -fy * ty * iz * iz;
    float m0[3] = {f.rot0[0] * s0 + f.rot2[0] * s1, f.rot0[1] * s0 + f.rot2[1] * s1, f.rot0[2] * s0 + f.rot2[2] * s1};
    float m1[3] = {f.rot1[0] * s2 + f.rot2[0] * s3, f.rot1[1] * s2 + f.rot2[1] * s3, f.rot1[2] * s2 + f.rot2[2] * s3};
    float c0[3], c1[3], c2[3];
    rot_cols(g2, c0, c1, c2);
    float sx = gx::exp(F_(2.0) * g1.x), sy = gx::exp(F_(2.0) * g1.y), sz = gx::exp(F_(2.0) * g1.z);
    float u0 = dot3(m0[0], m0[1], m0[2], c0[0], c0[1], c0[2]);
    float u1 = dot3(m0[0], m0[1], m0[2], c1[0], c1[1], c1[2]);
    float u2 = dot3(m0[0], m0[1], m0[2], c2[0], c2[1], c2[2]);
    float v0 = dot3(m1[0], m1[1], m1[2], c0[0], c0[1], c0[2]);
    float v1 = dot3(m1[0], m1[1], m1[2], c1[0], c1[1], c1[2]);
    float v2 = dot3(m1[0], m1[1], m1[2], c2[0], c2[1], c2[2]);
    float a = dot3(sx, sy, sz, u0 * u0, u1 * u1, u2 * u2) + f.low_pass;
    float b = dot3(sx, sy, sz, u0 * v0, u1 * v1, u2 * v2);
    float c = dot3(sx, sy, sz, v0 * v0, v1 * v1, v2 * v2) + f.low_pass;
    float det = a * c - b * b;
    if (!(det > F_(0.0))) return pr;
    pr.ok = true;
    pr.mx = div_(fx * cx, cz) + f.cx;
    pr.my = div_(fy * cy, cz) + f.cy;
    pr.a = a;
    pr.b = b;
    pr.c = c;
    pr.depth = cz;
    return pr;
}

// dilog (gps_splat.wgsl:79-94)
__device__ inline float dilog_series(float x) {
    float term = x, sum = x;
    for (uint32_t k = 2; k < 32; ++k) {
        term = term * x;
        sum = sum + div_(term, (float)(k * k));
    }
    return sum;
}
__device__ inline float dilog(float x) {
    if (x >= F_(1.0)) return gxc::kDilogOne;
    if (x <= F_(0.0)) return F_(0.0);
    if (x <= F_(0.5)) return dilog_series(x);
    return gxc::kDilogOne - gx::log(x) * gx::log(F_(1.0) - x) - dilog_series(F_(1.0) - x);
}
// inv_dilog / corrected_radius (gps_splat.wgsl:97-140), Li2(o) precomputed per splat
__device__ inline float inv_dilog(float tgt, float hi_in) {
    if (tgt <= F_(0.0)) return F_(0.0);
    float lo = F_(0.0), hi = hi_in, y = hi * F_(0.5);
    for (uint32_t i = 0; i < 24; ++i) {
        float f = dilog(y) - tgt;
        if (f > F_(0.0)) hi = y; else lo = y;
        float dfdy = F_(1.0);
        if (y > F_(1e-6) && y < F_(0.9999999)) dfdy = div_(-gx::log(F_(1.0) - y), y);
        float ny = y - div_(f, dfdy);
        if (!(ny > lo && ny < hi)) ny = F_(0.5) * (lo + hi);
        if (fabsf(ny - y) <= F_(1e-6) * (F_(1.0) + y)) return ny;
        y = ny;
    }
    return y;
}
__device__ inline float corrected_radius_exact(float o, float li2o, float u) {
    if (o <= F_(0.0)) return F_(0.0);
    float tgt = (F_(1.0) - u) * li2o;
    float y = fmin_(inv_dilog(tgt, o), o);
    if (y <= F_(0.0)) return F_(40.0);
    return sqrt_(fmax_(-F_(2.0) * gx::log(div_(y, o)), F_(0.0)));
}
__device__ __forceinline__ float mix_(float a, float b, float t) { return a * (F_(1.0) - t) + b * t; }
// corrected_radius_lut (gps_splat.wgsl:117-130) with the o-row (i0, a) hoisted per splat
__device__ __forceinline__ float corrected_radius_lut(const float* lut, uint32_t i0, float a, float u,
                                                     const float* lg = gx::tab_log()) {
    float v = -gx::log_t_pos(fmax_(F_(1.0) - u, gxc::kUMin), lg);
    float fv = fmin_(sqrt_(v) * gxc::kLutFv, F_(128.0));
    uint32_t j0 = min(f2u(fv), 127u);
    float b = fv - (float)j0;
    uint32_t k = i0 * 129u + j0;
    float r0 = mix_(lut[k], lut[k + 1], b);
    float r1 = mix_(lut[k + 129], lut[k + 130], b);
    return mix_(r0, r1, a);
}

// poisson (gps_splat.wgsl:142-160)
__device__ inline uint32_t poisson(float lambda, uint32_t* st) {
    if (lambda <= F_(0.0)) return 0u;
    if (lambda < F_(30.0)) {
        float l = gx::exp(-lambda);
        uint32_t k = 0;
        float p = F_(1.0);
        for (;;) {
            k = k + 1u;
            p = p * gx::next_u(st);
            if (p <= l) break;
        }
        return k - 1u;
    }
    float u1 = fmax_(gx::next_u(st), gxc::kUMin);
    float u2 = gx::next_u(st);
    float z = sqrt_(-F_(2.0) * gx::log(u1)) * gx::cos(gxc::kTwoPi * u2);
    return f2u(fmax_(gx::rint_(lambda + sqrt_(lambda) * z), F_(0.0)));
}

// extinction_term / pixel_density_scale / extinction_over_linear (gps_splat.wgsl:417-433)
__device__ inline float extinction_term(float o) {
    float c = fmin_(o, gxc::kOneMinus1e6);
    if (c < F_(1e-3)) return c * (F_(1.0) + c * (F_(0.5) + c * F_(0.33333334)));
    return -gx::log(F_(1.0) - c);
}
__device__ inline float pixel_density_scale(const FrameConst& f, float depth) {
    if (!(depth > fmax_(f.near_z, F_(0.0)))) return F_(0.0);
    float ratio = div_(f.refl, depth);
    return fmin_(ratio * ratio * f.fx * f.fy, F_(1.0e12));
}
__device__ __forceinline__ float eol(float x, const float* lg = gx::tab_log()) {
    if (x < F_(1e-4)) return F_(1.0) + F_(0.5) * x;
    return div_(-gx::log_t_pos(F_(1.0) - fmin_(x, gxc::kOneMinus1e6), lg), x);  // argument >= 1e-6
}

// splat_colour (gps_splat.wgsl:210-251)
__device__ inline float4 splat_colour(const FrameConst& f, const float* __restrict__ sh, uint32_t id, float4 g0, float4 g3) {
    float base[3] = {g3.x, g3.y, g3.z};
    uint32_t deg = f.sh_deg;
    if (deg == 0u) return make_float4(fmax_(base[0], F_(0.0)), fmax_(base[1], F_(0.0)), fmax_(base[2], F_(0.0)), F_(0.0));
    float dx = g0.x - f.pos[0], dy = g0.y - f.pos[1], dz = g0.z - f.pos[2];
    float len = sqrt_(dot3(dx, dy, dz, dx, dy, dz));
    float x = div_(dx, len), y = div_(dy, len), z = div_(dz, len);
    uint32_t r = f.sh_stride;
    const float* s = sh + (size_t)id * 3u * r;
    float out[3];
#pragma unroll
    for (int ch = 0; ch < 3; ++ch) {
        const float* S = s + ch * r;
        float acc = base[ch];
        acc = acc - F_(0.4886025119029199) * y * S[0] + F_(0.4886025119029199) * z * S[1] - F_(0.4886025119029199) * x * S[2];
        if (deg >= 2u) {
            float xx = x * x, yy = y * y, zz = z * z, xy = x * y, yz = y * z, xz = x * z;
            acc = acc + F_(1.0925484305920792) * xy * S[3] - F_(1.0925484305920792) * yz * S[4] +
                  F_(0.31539156525252005) * (F_(2.0) * zz - xx - yy) * S[5] - F_(1.0925484305920792) * xz * S[6] +
                  F_(0.5462742152960396) * (xx - yy) * S[7];
            if (deg >= 3u) {
                acc = acc - F_(0.5900435899266435) * y * (F_(3.0) * xx - yy) * S[8] + F_(2.890611442640554) * xy * z * S[9] -
                      F_(0.4570457994644658) * y * (F_(4.0) * zz - xx - yy) * S[10] +
                      F_(0.3731763325901154) * z * (F_(2.0) * zz - F_(3.0) * xx - F_(3.0) * yy) * S[11] -
                      F_(0.4570457994644658) * x * (F_(4.0) * zz - xx - yy) * S[12] +
                      F_(1.445305721320277) * z * (xx - yy) * S[13] - F_(0.5900435899266435) * x * (xx - F_(3.0) * yy) * S[14];
            }
        }
        out[ch] = fmax_(acc, F_(0.0));
    }
    return make_float4(out[0], out[1], out[2], F_(0.0));
}

}  // namespace gpsb
